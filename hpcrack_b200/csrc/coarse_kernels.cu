// The coarsest level's smoother in one thread block: pcg_u (mechanical_pcg.cpp:223-330) with all
// of its iterations - Dirichlet values, residual, direction, K p, dots, updates - in one launch,
// the level's vectors and element forces held in shared memory.  The V-cycle calls the coarsest
// solve once per cycle with 50 iterations (mechanical_multigrid.cpp:29-32); on a 9^3 level the
// multi-kernel smoother spends its time in launch and grid-synchronisation latency (three
// dependent kernels per iteration), which this kernel replaces by block barriers.
//
// Element forces are computed element-parallel into a shared buffer and gathered per node in a
// fixed order (no atomics): results are deterministic; their rounding differs from the strip
// kernels' only in the order of the same sums.
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "internal.h"

namespace hpc {
namespace {

constexpr int kCoarseThreads = 512;

struct CoarseArgs {
  LevelGeo g;
  double* u;
  const double* fu;
  double* ru;
  const double* invM;
  const double* Ke;
  const double* Ge;
  double Ut;
  int nb;
  double* scal;
  int s_rnorm;
};

// Sum over the block in a fixed order (warp trees, then the warps' sums in warp order).
__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) red[32] = t;
  }
  __syncthreads();
  return red[32];
}

__global__ void __launch_bounds__(kCoarseThreads, 1) coarse_pcg_kernel(CoarseArgs a) {
  extern __shared__ __align__(16) double csm[];
  const LevelGeo& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int N = nx * ny * nz, ex = nx - 1, ey = ny - 1, ez = nz - 1, E = ex * ey * ez;
  double* su = csm;          // 3N
  double* sr = su + 3 * N;   // 3N
  double* sp = sr + 3 * N;   // 3N
  double* sw = sp + 3 * N;   // 3N
  double* sm = sw + 3 * N;   // 3N inverse diagonal
  double* sK = sm + 3 * N;   // E element moduli (times the Gauss weight, 1/h^2 folded when isotropic)
  double* sG = sK + E;       // E
  double* sf = sG + E;       // 24 E element forces [m*8+n][e]
  double* red = sf + 24 * E; // 33
  const int tid = threadIdx.x, nt = blockDim.x;
  const bool iso = g.hx == g.hy && g.hy == g.hz;
  const SF s = make_sf(g);
  const double wg = iso ? g.wg * (s.ih[0] * s.ih[0]) : g.wg;

  // ---- load the level (dense layout in shared memory) and set the Dirichlet values (Dirichlet_BD)
  for (int q = tid; q < N; q += nt) {
    const int i = q % nx, j = (q / nx) % ny, k = q / (nx * ny);
    const long long n = nidx(g, i, j, k);
    const BcFlags bc = bc_flags(g, i, j, k);
    const bool fix[3] = {bc.c0, bc.c1, bc.c2};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double uv = a.u[n + m * g.n];
      if (fix[m]) uv = (m == 2 && bc.top) ? a.Ut : 0.0;
      su[m * N + q] = uv;
      sm[m * N + q] = a.invM[n + m * g.n];
      sp[m * N + q] = 0.0;
    }
  }
  for (int e = tid; e < E; e += nt) {
    const int i = e % ex, j = (e / ex) % ey, k = e / (ex * ey);
    const long long n = nidx(g, i, j, k);
    sK[e] = a.Ke[n] * wg;
    sG[e] = a.Ge[n] * wg;
  }
  __syncthreads();

  // element forces of the field v into sf, then gathered per node into out (fixed order)
  auto apply = [&](const double* v, double* out) {
    for (int e = tid; e < E; e += nt) {
      const int i = e % ex, j = (e / ex) % ey, k = e / (ex * ey);
      double uu[3][8], Kw[8], Gw[8], f[3][8];
#pragma unroll
      for (int n = 0; n < 8; ++n) {
        const int q = (i + (n & 1)) + (j + ((n >> 1) & 1)) * nx + (k + (n >> 2)) * nx * ny;
#pragma unroll
        for (int m = 0; m < 3; ++m) uu[m][n] = v[m * N + q];
        Kw[n] = sK[e];
        Gw[n] = sG[e];
      }
      if (iso)
        mech_element<true>(uu, Kw, Gw, s, f);
      else
        mech_element<false>(uu, Kw, Gw, s, f);
#pragma unroll
      for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int n = 0; n < 8; ++n) sf[(m * 8 + n) * E + e] = f[m][n];
    }
    __syncthreads();
    for (int q = tid; q < N; q += nt) {
      const int i = q % nx, j = (q / nx) % ny, k = q / (nx * ny);
      double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int n = 0; n < 8; ++n) {  // the element whose corner n is this node
        const int a0 = n & 1, b0 = (n >> 1) & 1, c0 = n >> 2;
        const int ei = i - a0, ej = j - b0, ek = k - c0;
        if (ei < 0 || ej < 0 || ek < 0 || ei >= ex || ej >= ey || ek >= ez) continue;
        const int e = ei + ej * ex + ek * ex * ey;
#pragma unroll
        for (int m = 0; m < 3; ++m) acc[m] += sf[(m * 8 + n) * E + e];
      }
#pragma unroll
      for (int m = 0; m < 3; ++m) out[m * N + q] = acc[m];
    }
    __syncthreads();
  };

  // ---- Initial residual r = f - K u, zero on Dirichlet rows; rz = (r, M^-1 r)
  apply(su, sw);
  double rz = 0.0, rn = 0.0;
  for (int q = tid; q < N; q += nt) {
    const int i = q % nx, j = (q / nx) % ny, k = q / (nx * ny);
    const long long n = nidx(g, i, j, k);
    const BcFlags bc = bc_flags(g, i, j, k);
    const bool fix[3] = {bc.c0, bc.c1, bc.c2};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const double rv = fix[m] ? 0.0 : a.fu[n + m * g.n] - sw[m * N + q];
      sr[m * N + q] = rv;
      rz = fma(rv, rv * sm[m * N + q], rz);
      rn = fma(rv, rv, rn);
    }
  }
  rz = block_sum(rz, red);
  rn = block_sum(rn, red);
  if (tid == 0 && a.s_rnorm >= 0) a.scal[a.s_rnorm] = rn;

  double rz_prev = 1.0;
  for (int it = 0; it < a.nb; ++it) {
    const double beta = it == 0 ? 0.0 : rz / rz_prev;
    for (int q = tid; q < 3 * N; q += nt) {
      const double z = sr[q] * sm[q];
      sp[q] = it == 0 ? z : fma(beta, sp[q], z);
    }
    __syncthreads();
    apply(sp, sw);
    double pw = 0.0;
    for (int q = tid; q < 3 * N; q += nt) pw = fma(sp[q], sw[q], pw);
    pw = block_sum(pw, red);
    const double alpha = rz / pw;
    double rz_new = 0.0;
    for (int q = tid; q < N; q += nt) {
      const int i = q % nx, j = (q / nx) % ny, k = q / (nx * ny);
      const BcFlags bc = bc_flags(g, i, j, k);
      const bool fix[3] = {bc.c0, bc.c1, bc.c2};
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const int o = m * N + q;
        su[o] = fma(sp[o], alpha, su[o]);
        const double rv = fix[m] ? 0.0 : fma(-sw[o], alpha, sr[o]);
        sr[o] = rv;
        rz_new = fma(rv, rv * sm[o], rz_new);
      }
    }
    rz_prev = rz;
    rz = block_sum(rz_new, red);
  }

  // ---- write u and the last residual back
  for (int q = tid; q < N; q += nt) {
    const int i = q % nx, j = (q / nx) % ny, k = q / (nx * ny);
    const long long n = nidx(g, i, j, k);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      a.u[n + m * g.n] = su[m * N + q];
      a.ru[n + m * g.n] = sr[m * N + q];
    }
  }
}

size_t coarse_smem_bytes(const LevelGeo& g) {
  const size_t N = (size_t)g.nx * g.ny * g.nz, E = (size_t)(g.nx - 1) * (g.ny - 1) * (g.nz - 1);
  return sizeof(double) * (15 * N + 26 * E + 33);
}

}  // namespace

bool coarse_pcg_fits(hpc_ctx* c, int level) {
  if (level == c->maxlevel) return false;  // the finest level's material is nodal, not element-constant
  return coarse_pcg_fits_geo(c->L[level]);
}
bool coarse_pcg_fits_geo(const LevelGeo& g) { return coarse_smem_bytes(g) <= 220 * 1024; }

// Shared-memory opt-in of the kernel on the current device (called by hpc_create).
int coarse_pcg_prepare() {
  HPC_CUDA(cudaFuncSetAttribute(coarse_pcg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
  return HPC_OK;
}

int launch_coarse_pcg_on(hpc_ctx* c, const LevelGeo& g, double* u, const double* fu, double* ru, const double* invM,
                         const double* Ke, const double* Ge, double Ut, int nb) {
  const size_t smem = coarse_smem_bytes(g);
  CoarseArgs a{g, u, fu, ru, invM, Ke, Ge, Ut, nb, c->scal, S_RNORM};
  coarse_pcg_kernel<<<1, kCoarseThreads, smem, c->stream>>>(a);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

int launch_coarse_pcg(hpc_ctx* c, int level, double Ut, int nb) {
  const LevelFields& F = c->F[level];
  return launch_coarse_pcg_on(c, c->L[level], F.u, F.fu, F.ru, F.preMu, F.Ke, F.Ge, Ut, nb);
}

}  // namespace hpc
