// Vector, transfer, boundary-condition, material and history kernels.  All are HBM-bound
// streaming kernels over one or two levels; those that produce a global scalar use the
// deterministic grid reduction of device_common.cuh.
#include <cuda_runtime.h>

#include <algorithm>

#include "device_common.cuh"
#include "internal.h"

namespace hpc {

namespace {

int num_sms_v() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

// Node-parallel launch: a grid-stride loop over the nx*ny*nz nodes of a level (flat, x fastest,
// so neighbouring threads touch neighbouring addresses), at most 8 blocks of 256 threads per SM.
constexpr int kRowThreads = 256;
int row_grid(const LevelGeo& g, int per_sm = 8) {
  const long long nodes = (long long)g.nx * g.ny * g.nz;
  const long long blocks = (nodes + kRowThreads - 1) / kRowThreads;
  const long long cap = (long long)num_sms_v() * per_sm;
  return (int)(blocks < cap ? blocks : cap);
}

// Level sizes stay below 2^31 nodes (hpc_create checks), so 32-bit index arithmetic suffices.  The
// inner one-pass loop declares the node coordinates (i, j, kz) for the body; `continue` in the body
// moves on to the next node.
#define FOR_NODES(g)                                                                                 \
  for (unsigned _f = blockIdx.x * blockDim.x + threadIdx.x, _nodes = (unsigned)((g).nx * (g).ny * (g).nz); \
       _f < _nodes; _f += gridDim.x * blockDim.x)                                                     \
    for (int i = (int)(_f % (unsigned)(g).nx), j = (int)((_f / (unsigned)(g).nx) % (unsigned)(g).ny),    \
             kz = (int)(_f / ((unsigned)(g).nx * (unsigned)(g).ny)), _once = 1;                        \
         _once; _once = 0)

}  // namespace

// ---------------------------------------------------------------------------------------------
// PCG updates (mechanical_pcg.cpp:301-321, phase_field_pcg.cpp:192-200)
// ---------------------------------------------------------------------------------------------
// Two x-adjacent slots per thread with 16-byte accesses over the padded layout (the x pitch is a
// multiple of 4, so a pair never straddles a row; padding slots hold zeros in u, r, p, w and invM
// and stay zero).  Dirichlet flags exist only on the bottom and top planes.
template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// SLAB: sums over owned planes only (a z-slab context); the whole-specimen instance keeps the register
// budget of the plain loop (48 against 58 with the test).
template <typename T, bool SLAB = false>
__global__ void mech_update_kernel(LevelGeo g, T* u, T* r, const T* p, const T* w, const T* invM, int s_rz, int s_pw,
                                   RedTarget red) {
  using V2 = typename Vec2<T>::type;
  const T alpha = (T)(red.scal[s_rz] / red.scal[s_pw]);
  double rz = 0.0, rn = 0.0;
  const unsigned half = (unsigned)g.px / 2u, npairs = half * (unsigned)g.ny * (unsigned)g.nz;
  for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < npairs; q += gridDim.x * blockDim.x) {
    const unsigned row = q / half;  // j + k * ny
    const int i = 2 * (int)(q - row * half);
    const int kz = (int)(row / (unsigned)g.ny), j = (int)(row - (unsigned)kz * (unsigned)g.ny);
    const long long n = (long long)row * g.px + i;
    const double rz0 = rz, rn0 = rn;
    bool fix[2][3] = {{false, false, false}, {false, false, false}};
    if (g.bz[kz]) {
#pragma unroll
      for (int h = 0; h < 2; ++h)
        if (i + h < g.nx) {
          const BcFlags bc = bc_flags(g, i + h, j, kz);
          fix[h][0] = bc.c0;
          fix[h][1] = bc.c1;
          fix[h][2] = bc.c2;
        }
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const long long o = n + (long long)m * g.n;
      const V2 pv = *reinterpret_cast<const V2*>(p + o);
      const V2 wv = *reinterpret_cast<const V2*>(w + o);
      const V2 mv = *reinterpret_cast<const V2*>(invM + o);
      V2 uv = *reinterpret_cast<const V2*>(u + o);
      V2 rv = *reinterpret_cast<const V2*>(r + o);
      uv.x = fma(pv.x, alpha, uv.x);
      uv.y = fma(pv.y, alpha, uv.y);
      rv.x = fix[0][m] ? T(0) : fma(-wv.x, alpha, rv.x);
      rv.y = fix[1][m] ? T(0) : fma(-wv.y, alpha, rv.y);
      *reinterpret_cast<V2*>(u + o) = uv;
      *reinterpret_cast<V2*>(r + o) = rv;
      rz = fma((double)rv.x, (double)(rv.x * mv.x), rz);
      rz = fma((double)rv.y, (double)(rv.y * mv.y), rz);
      rn = fma((double)rv.x, (double)rv.x, rn);
      rn = fma((double)rv.y, (double)rv.y, rn);
    }
    if (SLAB && !owned_plane(g, kz)) {  // a ghost plane adds nothing (its values may be anything)
      rz = rz0;
      rn = rn0;
    }
  }
  double v[3] = {rz, rn, 0.0};
  grid_reduce<3>(v, red);
}

int launch_mech_update_on(hpc_ctx* c, int level, double* x, double* r, const double* p, const double* w,
                          const double* invM, int s_num, int s_den, int s_rz_next, int s_rn) {
  const LevelGeo& g = c->L[level];
  const long long pairs = (long long)(g.px / 2) * g.ny * g.nz;
  const int grid = (int)std::min<long long>((pairs + kRowThreads - 1) / kRowThreads, (long long)num_sms_v() * 8);
  const int cls = level == c->maxlevel ? HPC_KC_MECH_UPDATE_FINEST : HPC_KC_NONE;
  timing_begin(c, cls);
  if (c->slab)
    mech_update_kernel<double, true><<<grid, kRowThreads, 0, c->stream>>>(g, x, r, p, w, invM, s_num, s_den,
                                                                        make_red(c, s_rz_next, s_rn, -1));
  else
    mech_update_kernel<double, false><<<grid, kRowThreads, 0, c->stream>>>(g, x, r, p, w, invM, s_num, s_den,
                                                                         make_red(c, s_rz_next, s_rn, -1));
  timing_end(c, cls);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

int launch_mech_update(hpc_ctx* c, int level, const double* p, int s_rz, int s_pw, int s_rz_next, int s_rn) {
  const LevelFields& F = c->F[level];
  return launch_mech_update_on(c, level, F.u, F.ru, p, F.w, F.preMu, s_rz, s_pw, s_rz_next, s_rn);
}

// ---------------------------------------------------------------------------------------------
// Flexible PCG of the precision form: two dot products in one pass, the flexible direction update
// ---------------------------------------------------------------------------------------------
// TA = float: the precision form's z straight from the FP32 V-cycle (its FP64 copy is exact, so the
// sums are the same bits without the conversion pass).
template <typename TA>
__global__ void dot2_kernel(LevelGeo g, const TA* a, const double* b, const double* cv, RedTarget red) {
  double s0 = 0.0, s1 = 0.0;
  FOR_NODES(g) {
    if (!owned_plane(g, kz)) continue;
    const long long n = nidx(g, i, j, kz);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const long long o = n + (long long)m * g.n;
      const double av = (double)a[o];
      s0 = fma(av, b[o], s0);
      if (cv) s1 = fma(av, cv[o], s1);
    }
  }
  double v[2] = {s0, s1};
  grid_reduce<2>(v, red);
}

template <typename TA>
static int launch_dot2_t(hpc_ctx* c, int level, const TA* a, const double* b, const double* cv, int s0, int s1) {
  const LevelGeo& g = c->L[level];
  dot2_kernel<TA><<<row_grid(g), kRowThreads, 0, c->stream>>>(g, a, b, cv, make_red(c, s0, cv ? s1 : -1, -1));
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}
int launch_dot2(hpc_ctx* c, int level, const double* a, const double* b, const double* cv, int s0, int s1) {
  return launch_dot2_t(c, level, a, b, cv, s0, s1);
}
int launch_dot2(hpc_ctx* c, int level, const float* a, const double* b, const double* cv, int s0, int s1) {
  return launch_dot2_t(c, level, a, b, cv, s0, s1);
}

template <typename TZ>
__global__ void fcg_dir_kernel(LevelGeo g, const TZ* z, double* p, int first, const double* scal, int s_delta,
                               int s_gamma, int s_delta_prev) {
  const double beta = first ? 0.0 : (scal[s_delta] - scal[s_gamma]) / scal[s_delta_prev];
  FOR_NODES(g) {
    const long long n = nidx(g, i, j, kz);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const long long o = n + (long long)m * g.n;
      const double zv = (double)z[o];
      p[o] = first ? zv : fma(beta, p[o], zv);
    }
  }
}

template <typename TZ>
static int launch_fcg_dir_t(hpc_ctx* c, int level, const TZ* z, double* p, bool first, int s_delta, int s_gamma,
                            int s_delta_prev) {
  const LevelGeo& g = c->L[level];
  fcg_dir_kernel<TZ><<<row_grid(g), kRowThreads, 0, c->stream>>>(g, z, p, first ? 1 : 0, c->scal, s_delta, s_gamma,
                                                                s_delta_prev);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, level, p, 3, sizeof(double));  // the apply of p reads its ghost planes
  return HPC_OK;
}
int launch_fcg_dir(hpc_ctx* c, int level, const double* z, double* p, bool first, int s_delta, int s_gamma,
                   int s_delta_prev) {
  return launch_fcg_dir_t(c, level, z, p, first, s_delta, s_gamma, s_delta_prev);
}
int launch_fcg_dir(hpc_ctx* c, int level, const float* z, double* p, bool first, int s_delta, int s_gamma,
                   int s_delta_prev) {
  return launch_fcg_dir_t(c, level, z, p, first, s_delta, s_gamma, s_delta_prev);
}

__global__ void pf_update_kernel(LevelGeo g, double* d, double* r, const double* p, const double* w,
                                 const double* invM, int s_rz, int s_pw, RedTarget red) {
  const double alpha = red.scal[s_rz] / red.scal[s_pw];
  double rz = 0.0, rn = 0.0;
  FOR_NODES(g) {
    const long long n = nidx(g, i, j, kz);
    d[n] = fma(p[n], alpha, d[n]);
    const double rv = fma(-w[n], alpha, r[n]);
    r[n] = rv;
    const bool own = owned_plane(g, kz);
    const double z1 = fma(rv, rv * invM[n], rz), n1 = fma(rv, rv, rn);
    rz = own ? z1 : rz;
    rn = own ? n1 : rn;
  }
  double v[3] = {rz, rn, 0.0};
  grid_reduce<3>(v, red);
}

int launch_pf_update(hpc_ctx* c, int level, const double* p, int s_rz, int s_pw, int s_rz_next, int s_rn) {
  const LevelGeo& g = c->L[level];
  const LevelFields& F = c->F[level];
  pf_update_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(g, F.d, F.R, p, F.wd, F.preMd, s_rz, s_pw,
                                                              make_red(c, s_rz_next, s_rn, -1));
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// PCG direction (mechanical_pcg.cpp:274-292, phase_field_pcg.cpp:178-186):
// z = r M^-1, beta = rz/rz_old (0 on a call's first iteration), p = z + beta p, in place.
template <typename T>
__global__ void dir_update_kernel(LevelGeo g, int ncomp, const T* r, const T* invM, T* p, int first,
                                  const double* scal, int s_rz, int s_rz_prev) {
  const T beta = first ? T(0) : (T)(scal[s_rz] / scal[s_rz_prev]);
  FOR_NODES(g) {
    const long long n = nidx(g, i, j, kz);
    for (int m = 0; m < ncomp; ++m) {
      const long long o = n + (long long)m * g.n;
      const T z = r[o] * invM[o];
      p[o] = first ? z : fma(beta, p[o], z);
    }
  }
}
int launch_dir_update(hpc_ctx* c, int level, int ncomp, const double* r, const double* invM, double* p, bool first,
                      int s_rz, int s_rz_prev) {
  const LevelGeo& g = c->L[level];
  dir_update_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(g, ncomp, r, invM, p, first ? 1 : 0, c->scal, s_rz,
                                                               s_rz_prev);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, level, p, ncomp, sizeof(double));  // SendRecv(z), mechanical_pcg.cpp:278, phase_field_pcg.cpp:180
  return HPC_OK;
}

// ---------------------------------------------------------------------------------------------
// Dirichlet conditions (boundary_conditions.cpp:20-154) on the planes that carry any flag
// ---------------------------------------------------------------------------------------------
template <typename T>
__global__ void bc_kernel(LevelGeo g, T* v, const T* src, int kind, T Ut) {
  FOR_NODES(g) {
    if (g.bz[kz] == 0) continue;
    const BcFlags bc = bc_flags(g, i, j, kz);
    const long long n = nidx(g, i, j, kz);
    if (kind == 0) {
      if (bc.c0) v[n] = T(0);
      if (bc.c1) v[n + g.n] = T(0);
      if (bc.c2) v[n + 2 * g.n] = bc.top ? Ut : T(0);
    } else if (kind == 1) {
      if (bc.c0) v[n] = src[n];
      if (bc.c1) v[n + g.n] = src[n + g.n];
      if (bc.c2) v[n + 2 * g.n] = src[n + 2 * g.n];
    } else {
      if (bc.c0) v[n] = T(0);
      if (bc.c1) v[n + g.n] = T(0);
      if (bc.c2) v[n + 2 * g.n] = T(0);
    }
  }
}

int launch_bc(hpc_ctx* c, int level, double* v, const double* src, int kind, double Ut) {
  const LevelGeo& g = c->L[level];
  bc_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(g, v, src, kind, Ut);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// ---------------------------------------------------------------------------------------------
// dots and helpers
// ---------------------------------------------------------------------------------------------
__global__ void dot_kernel(LevelGeo g, int ncomp, const double* a, const double* b, RedTarget red) {
  double s = 0.0;
  FOR_NODES(g) {
    if (!owned_plane(g, kz)) continue;
    const long long n = nidx(g, i, j, kz);
    for (int m = 0; m < ncomp; ++m) {
      const long long o = n + (long long)m * g.n;
      s = fma(a[o], b ? b[o] : a[o], s);
    }
  }
  double v[1] = {s};
  grid_reduce<1>(v, red);
}

int launch_dot(hpc_ctx* c, int level, int ncomp, const double* a, const double* b, int slot) {
  const LevelGeo& g = c->L[level];
  dot_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(g, ncomp, a, b, make_red(c, slot, -1, -1));
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

__global__ void fill_kernel(double* v, long long n, double value) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v[i] = value;
}
int launch_fill(hpc_ctx* c, double* v, long long n, double value) {
  long long blocks = (n + 255) / 256;
  int grid = (int)(blocks < num_sms_v() * 16LL ? blocks : num_sms_v() * 16LL);
  if (grid <= 0) return HPC_OK;
  fill_kernel<<<grid, 256, 0, c->stream>>>(v, n, value);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

__global__ void invert_kernel(LevelGeo g, int ncomp, double* v) {
  FOR_NODES(g) {
    const long long n = nidx(g, i, j, kz);
    for (int m = 0; m < ncomp; ++m) v[n + m * g.n] = 1.0 / v[n + m * g.n];
  }
}
int launch_invert(hpc_ctx* c, int level, int ncomp, double* v) {
  const LevelGeo& g = c->L[level];
  invert_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(g, ncomp, v);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// The compute capability the library's device code was built for, as the runtime reports it for
// one of its kernels (major * 10 + minor; 100 for sm_100a).
cudaError_t kernel_binary_version(int* version) {
  cudaFuncAttributes a{};
  const cudaError_t e = cudaFuncGetAttributes(&a, invert_kernel);
  if (e == cudaSuccess) *version = a.binaryVersion;
  return e;
}

__global__ void axpby_kernel(double* y, const double* a, const double* b, double sa, double sb, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = sa * a[i] + (b ? sb * b[i] : 0.0);
}
int launch_axpby(hpc_ctx* c, double* y, const double* a, const double* b, double sa, double sb, long long n) {
  long long blocks = (n + 255) / 256;
  int grid = (int)(blocks < num_sms_v() * 16LL ? blocks : num_sms_v() * 16LL);
  if (grid <= 0) return HPC_OK;
  axpby_kernel<<<grid, 256, 0, c->stream>>>(y, a, b, sa, sb, n);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// ---------------------------------------------------------------------------------------------
// inter-grid transfers (multigrid_intergrid.cpp)
// ---------------------------------------------------------------------------------------------
// solution_injection (:25-90)
// On a z slab, coarse plane kc lies on fine plane 2 kc + zsh; a lower ghost plane without a fine
// plane below it is left to the ghost exchange that follows every transfer.
__global__ void inject_kernel(LevelGeo gc, LevelGeo gf, const double* f, double* co, int ncomp) {
  FOR_NODES(gc) {
    const int fz = 2 * kz + gc.zsh;
    if (fz < 0) continue;
    const long long nc = nidx(gc, i, j, kz), nf = nidx(gf, 2 * i, 2 * j, fz);
    for (int m = 0; m < ncomp; ++m) co[nc + m * gc.n] = f[nf + m * gf.n];
  }
}
int launch_inject(hpc_ctx* c, int lf, const double* f, double* co, int ncomp) {
  inject_kernel<<<row_grid(c->L[lf - 1]), kRowThreads, 0, c->stream>>>(c->L[lf - 1], c->L[lf], f, co, ncomp);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, lf - 1, co, ncomp, sizeof(double));
  return HPC_OK;
}

// coarsen_u (:106-121): inject, Dirichlet_BD on the coarse level, save uold.
template <typename T>
__global__ void inject_u_kernel(LevelGeo gc, LevelGeo gf, const T* uf, T* uc, T* uold, T Ut) {
  FOR_NODES(gc) {
    const int fz = 2 * kz + gc.zsh;
    if (fz < 0) continue;
    const long long nc = nidx(gc, i, j, kz), nf = nidx(gf, 2 * i, 2 * j, fz);
    T v[3] = {uf[nf], uf[nf + gf.n], uf[nf + 2 * gf.n]};
    if (gc.bz[kz]) {
      const BcFlags bc = bc_flags(gc, i, j, kz);
      if (bc.c0) v[0] = T(0);
      if (bc.c1) v[1] = T(0);
      if (bc.c2) v[2] = bc.top ? Ut : T(0);
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      uc[nc + m * gc.n] = v[m];
      uold[nc + m * gc.n] = v[m];
    }
  }
}
int launch_inject_u(hpc_ctx* c, int lf, double Ut) {
  inject_u_kernel<<<row_grid(c->L[lf - 1]), kRowThreads, 0, c->stream>>>(
      c->L[lf - 1], c->L[lf], c->F[lf].u, c->F[lf - 1].u, c->F[lf - 1].uold, Ut);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, lf - 1, c->F[lf - 1].u, 3, sizeof(double));  // SendRecv(uc), multigrid_intergrid.cpp:116
  HPC_SLAB_HALO(c, lf - 1, c->F[lf - 1].uold, 3, sizeof(double));
  return HPC_OK;
}

// coarsen_d (:92-103)
__global__ void inject_d_kernel(LevelGeo gc, LevelGeo gf, const double* df, double* dc, double* dold) {
  FOR_NODES(gc) {
    const int fz = 2 * kz + gc.zsh;
    if (fz < 0) continue;
    const long long nc = nidx(gc, i, j, kz), nf = nidx(gf, 2 * i, 2 * j, fz);
    const double v = df[nf];
    dc[nc] = v;
    dold[nc] = v;
  }
}
int launch_inject_d(hpc_ctx* c, int lf) {
  inject_d_kernel<<<row_grid(c->L[lf - 1]), kRowThreads, 0, c->stream>>>(c->L[lf - 1], c->L[lf], c->F[lf].d,
                                                                          c->F[lf - 1].d, c->F[lf - 1].dold);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, lf - 1, c->F[lf - 1].d, 1, sizeof(double));  // SendRecv(dc), multigrid_intergrid.cpp:99
  HPC_SLAB_HALO(c, lf - 1, c->F[lf - 1].dold, 1, sizeof(double));
  return HPC_OK;
}

// coarsen_f_standard_routine (:124-342), standalone form (full_weight in device_common.cuh).
__global__ void restrict_kernel(LevelGeo gc, LevelGeo gf, const double* rf, const double* Fic, double* fc, int ncomp) {
  FOR_NODES(gc) {
    const long long nc = nidx(gc, i, j, kz);
    const int fz = 2 * kz + gc.zsh;
    for (int m = 0; m < ncomp; ++m)
      fc[nc + m * gc.n] = Fic[nc + m * gc.n] + (fz >= 0 ? full_weight(gf, rf + m * gf.n, 2 * i, 2 * j, fz) : 0.0);
  }
}
int launch_restrict(hpc_ctx* c, int lf, const double* rf, const double* Fic, double* fc, int ncomp) {
  HPC_SLAB_HALO(c, lf, rf, ncomp, sizeof(double));  // SendRecv(rf), multigrid_intergrid.cpp:356,393
  restrict_kernel<<<row_grid(c->L[lf - 1]), kRowThreads, 0, c->stream>>>(c->L[lf - 1], c->L[lf], rf, Fic, fc, ncomp);
  HPC_CHECK_LAUNCH(c);
  // SendRecv(fc), :369,411.  (The solves' fused restriction skips it: there the coarse right-hand side
  // on ghost planes only feeds ghost residuals, which the next restriction takes from the neighbours.)
  HPC_SLAB_HALO(c, lf - 1, fc, ncomp, sizeof(double));
  return HPC_OK;
}

// refine_standard_routine (:416-520) as a gather over fine nodes, with the reference's term order;
// optionally followed by Dirichlet_BD on the fine level (refine_u, :536-549).
template <typename T>
__global__ void prolong_kernel(LevelGeo gc, LevelGeo gf, const T* uc, const T* ucold, T* uf, int ncomp, int apply_bc,
                               T Ut) {
  FOR_NODES(gf) {
    const int zq = kz - gc.zsh;  // fine plane counted from the coarse grid's plane 0
    const int ox = i & 1, oy = j & 1, oz = zq & 1;
    const int ic = (i + 1) >> 1, jc = (j + 1) >> 1, kc = (zq + 1) >> 1;
    const long long nf = nidx(gf, i, j, kz);
    BcFlags bc{false, false, false, false};
    if (apply_bc && gf.bz[kz]) bc = bc_flags(gf, i, j, kz);
    for (int m = 0; m < ncomp; ++m) {
      const T* a = uc + m * gc.n;
      const T* o = ucold + m * gc.n;
      auto E = [&](int x, int y, int z) -> T {
        const long long q = nidx(gc, x, y, z);
        return a[q] - o[q];
      };
      T add;
      if (!ox && !oy && !oz) add = E(ic, jc, kc);
      else if (ox && !oy && !oz) add = T(0.5) * (E(ic, jc, kc) + E(ic - 1, jc, kc));
      else if (!ox && oy && !oz) add = T(0.5) * (E(ic, jc, kc) + E(ic, jc - 1, kc));
      else if (!ox && !oy && oz) add = T(0.5) * (E(ic, jc, kc) + E(ic, jc, kc - 1));
      else if (ox && oy && !oz)
        add = T(0.25) * (E(ic, jc, kc) + E(ic, jc - 1, kc) + E(ic - 1, jc, kc) + E(ic - 1, jc - 1, kc));
      else if (ox && !oy && oz)
        add = T(0.25) * (E(ic, jc, kc) + E(ic - 1, jc, kc - 1) + E(ic, jc, kc - 1) + E(ic - 1, jc, kc));
      else if (!ox && oy && oz)
        add = T(0.25) * (E(ic, jc, kc) + E(ic, jc - 1, kc - 1) + E(ic, jc, kc - 1) + E(ic, jc - 1, kc));
      else
        add = T(0.125) * (E(ic, jc, kc) + E(ic, jc - 1, kc) + E(ic - 1, jc, kc) + E(ic - 1, jc - 1, kc) +
                          E(ic, jc, kc - 1) + E(ic - 1, jc, kc - 1) + E(ic, jc - 1, kc - 1) + E(ic - 1, jc - 1, kc - 1));
      T v = uf[nf + m * gf.n] + add;
      if (apply_bc) {
        if (m == 0 && bc.c0) v = T(0);
        if (m == 1 && bc.c1) v = T(0);
        if (m == 2 && bc.c2) v = bc.top ? Ut : T(0);
      }
      uf[nf + m * gf.n] = v;
    }
  }
}
int launch_prolong(hpc_ctx* c, int lf, const double* uc, const double* ucold, double* uf, int ncomp, bool apply_bc,
                   double Ut) {
  prolong_kernel<<<row_grid(c->L[lf]), kRowThreads, 0, c->stream>>>(c->L[lf - 1], c->L[lf], uc, ucold, uf, ncomp,
                                                                     apply_bc ? 1 : 0, Ut);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, lf, uf, ncomp, sizeof(double));  // SendRecv(uf), multigrid_intergrid.cpp:531,547
  return HPC_OK;
}

// ---------------------------------------------------------------------------------------------
// material selection (material_selection.cpp) and coarse element material
// ---------------------------------------------------------------------------------------------
struct ChoiceK {
  LevelGeo g;
  const double *u, *bulK, *G, *d;
  int8_t* choice;
  double *Ke, *Ge;
  double small_k;
  int quirk, do_choice, do_element;
  int nzg;  // planes of the whole specimen on this level (a slab evaluates the quirk on global planes)
};

__device__ __forceinline__ void load8(const double* f, const LevelGeo& g, int i, int j, int k, double (&v)[8]) {
#pragma unroll
  for (int n = 0; n < 8; ++n) v[n] = f[nidx(g, i + (n & 1), j + ((n >> 1) & 1), k + (n >> 2))];
}

// MP_choice_element (:19-45) fused with MP_element (:67-98) for one element.
__global__ void choice_kernel(ChoiceK a) {
  const LevelGeo& g = a.g;
  const SF s = make_sf(g);
  for (long long row = blockIdx.x; row < (long long)(g.ny - 1) * (g.nz - 1); row += gridDim.x) {
    const int j = (int)(row % (g.ny - 1)), k = (int)(row / (g.ny - 1));
    for (int i = threadIdx.x; i < g.nx - 1; i += blockDim.x) {
      const long long e = nidx(g, i, j, k);
      double Kn[8], Gn[8], Kg[8], Gg[8];
      load8(a.bulK, g, i, j, k, Kn);
      load8(a.G, g, i, j, k, Gn);
      gp_material(Kn, s, Kg);
      gp_material(Gn, s, Gg);
      // the reference's loop bounds use the dense extent nx; the flat slot is i + j*nx + k*nx*ny, on the
      // whole specimen's planes, so that a z-split regime field equals the unsplit one
      const long long flat = (long long)i + (long long)j * g.nx + (long long)(g.zb + k) * g.nx * g.ny;
      int ch = 0;
      if (!a.do_choice) {
        ch = a.choice[e];
      } else if (!a.quirk || choice_in_image(flat, g.nx, g.ny, a.nzg)) {
        double gx[3][4], gy[3][4], gz[3][4];
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          double un[8];
          load8(a.u + m * g.n, g, i, j, k, un);
          sf_forward(un, s, gx[m], gy[m], gz[m], (double*)nullptr);
        }
        double tr = 0.0, pp = 0.0, pn = 0.0;
#pragma unroll
        for (int gp = 0; gp < 8; ++gp) {
          const Strain e8 = strain_at(gx, gy, gz, gp & 1, (gp >> 1) & 1, gp >> 2);
          tr += e8.xx + e8.yy + e8.zz;
          pp += phi_pos(Kg[gp], Gg[gp], e8);
          pn += phi_neg(Kg[gp], e8);
        }
        ch = tr >= 0.0 ? 0 : 1;
        if (pp < pn) ch = 2;
      }
      if (a.do_choice) a.choice[e] = (int8_t)ch;
      if (a.do_element) {
        double dn[8], dg[8];
        load8(a.d, g, i, j, k, dn);
        gp_material(dn, s, dg);
        double Ks = 0.0, Gs = 0.0;
#pragma unroll
        for (int gp = 0; gp < 8; ++gp) {
          const double dd = fmin(fmax(dg[gp], 0.0), 1.0);
          const double om = 1.0 - dd;
          const double gd = fma((1.0 - a.small_k) * om, om, a.small_k);
          Ks += ch == 0 ? gd * Kg[gp] : Kg[gp];
          Gs += ch == 2 ? Gg[gp] : gd * Gg[gp];
        }
        a.Ke[e] = 0.125 * Ks;
        a.Ge[e] = 0.125 * Gs;
      }
    }
  }
}

int launch_choice_level(hpc_ctx* c, int level, double small_k, bool do_choice, bool do_element) {
  const LevelGeo& g = c->L[level];
  const LevelFields& F = c->F[level];
  if (do_choice) HPC_CUDA(cudaMemsetAsync(F.choice, 0, (size_t)g.n, c->stream));
  if (g.nx < 2 || g.ny < 2 || g.nz < 2) return HPC_OK;
  ChoiceK a{g, F.u, F.bulK, F.G, F.d, F.choice, F.Ke, F.Ge, small_k, c->choice_quirk, do_choice ? 1 : 0,
            do_element ? 1 : 0, c->geo.element_nb[2] * (1 << level) + 1};
  long long rows = (long long)(g.ny - 1) * (g.nz - 1);
  int grid = (int)(rows < num_sms_v() * 8LL ? rows : num_sms_v() * 8LL);
  choice_kernel<<<grid, 128, 0, c->stream>>>(a);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

int launch_choice_element(hpc_ctx* c, double small_k, bool do_choice, bool do_element) {
  return launch_choice_level(c, c->maxlevel, small_k, do_choice, do_element);
}
int launch_mp_choice_level(hpc_ctx* c, int level) { return launch_choice_level(c, level, 0.0, true, false); }

// coarse_voigt / coarse_reuss (material_coarse_element.cpp:20-82); hill=1 gives VR_all_level's
// 0.5*(0.5*(V+R) + sqrt(V*R)) written over the whole coarse array (:96), hill=0 Voigt_all_level
// (element slots only, :112).
__global__ void vr_kernel(LevelGeo gc, LevelGeo gf, const double* Hf, double* Hc, int hill, int whole) {
  FOR_NODES(gc) {
    const long long nc = nidx(gc, i, j, kz);
    const bool elem = i <= gc.nx - 2 && j <= gc.ny - 2 && kz <= gc.nz - 2;
    if (!elem) {
      if (whole) Hc[nc] = 0.0;
      continue;
    }
    const int x = 2 * i, y = 2 * j, z = 2 * kz + gc.zsh;
    if (z < 0) continue;
    const double h[8] = {Hf[nidx(gf, x, y, z)],         Hf[nidx(gf, x + 1, y, z)],
                         Hf[nidx(gf, x, y + 1, z)],     Hf[nidx(gf, x + 1, y + 1, z)],
                         Hf[nidx(gf, x, y, z + 1)],     Hf[nidx(gf, x + 1, y, z + 1)],
                         Hf[nidx(gf, x, y + 1, z + 1)], Hf[nidx(gf, x + 1, y + 1, z + 1)]};
    const double V = 0.125 * (h[0] + h[1] + h[2] + h[3] + h[4] + h[5] + h[6] + h[7]);
    if (!hill) {
      Hc[nc] = V;
      continue;
    }
    const double Rr = 8. / (1. / h[0] + 1. / h[1] + 1. / h[2] + 1. / h[3] + 1. / h[4] + 1. / h[5] + 1. / h[6] + 1. / h[7]);
    Hc[nc] = 0.5 * (0.5 * (V + Rr) + sqrt(V * Rr));
  }
}
int launch_vr(hpc_ctx* c, int lf, const double* Hf, double* Hc, bool hill, bool whole_array) {
  vr_kernel<<<row_grid(c->L[lf - 1]), kRowThreads, 0, c->stream>>>(c->L[lf - 1], c->L[lf], Hf, Hc, hill ? 1 : 0,
                                                                    whole_array ? 1 : 0);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, lf - 1, Hc, 1, sizeof(double));  // SendRecv(H), material_coarse_element.cpp:98,114
  return HPC_OK;
}

// voight / reuss / coarse_VR (image_input.cpp:144-260): 27-point clamped means, Hill combination.
__global__ void coarse_vr_kernel(LevelGeo gc, LevelGeo gf, const double* f, double* co) {
  FOR_NODES(gc) {
    const int x = 2 * i, y = 2 * j, z = 2 * kz + gc.zsh;
    if (z < 0) continue;
    const int Xl = gf.nx - 1, Yl = gf.ny - 1, Zl = gf.nz - 1;
    const int xm = max(x - 1, 0), xp = min(x + 1, Xl), ym = max(y - 1, 0), yp = min(y + 1, Yl);
    const int zm = max(z - 1, 0), zp = min(z + 1, Zl);
    const int ax[27] = {xm, xm, xm, xm, xp, xp, xp, xp, xm, xm, xp, xp, xm, xm, xp, xp, x, x, x, x, x, x, x, x, xm, xp, x};
    const int ay[27] = {ym, ym, yp, yp, ym, ym, yp, yp, ym, yp, ym, yp, y, y, y, y, ym, ym, yp, yp, y, y, ym, yp, y, y, y};
    const int az[27] = {zm, zp, zm, zp, zm, zp, zm, zp, z, z, z, z, zm, zp, zm, zp, zm, zp, zm, zp, zm, zp, z, z, z, z, z};
    double v0 = f[nidx(gf, ax[0], ay[0], az[0])];
    double sv = v0, sr = 1. / v0;
    for (int q = 1; q < 27; ++q) {
      const double v = f[nidx(gf, ax[q], ay[q], az[q])];
      sv = sv + v;
      sr = sr + 1. / v;
    }
    const double mv = (1.0 / 27.0) * sv;
    const double mr = 27.0 / sr;
    co[nidx(gc, i, j, kz)] = 0.5 * (0.5 * (mv + mr) + sqrt(mv * mr));
  }
}
int launch_coarse_vr(hpc_ctx* c, int lf, const double* f, double* co) {
  coarse_vr_kernel<<<row_grid(c->L[lf - 1]), kRowThreads, 0, c->stream>>>(c->L[lf - 1], c->L[lf], f, co);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, lf - 1, co, 1, sizeof(double));  // SendRecv(MP), image_input.cpp:269
  return HPC_OK;
}

// ---------------------------------------------------------------------------------------------
// history, right-hand side, reductions
// ---------------------------------------------------------------------------------------------
// strain_history (strain_history.cpp:162-210)
__global__ void strain_history_kernel(LevelGeo g, const double* u, const double* bulK, const double* G,
                                      const double* gc, double* H, double lc, double uprop) {
  const SF s = make_sf(g);
  for (long long row = blockIdx.x; row < (long long)(g.ny - 1) * (g.nz - 1); row += gridDim.x) {
    const int j = (int)(row % (g.ny - 1)), k = (int)(row / (g.ny - 1));
    for (int i = threadIdx.x; i < g.nx - 1; i += blockDim.x) {
      double Kn[8], Gn[8], cn[8], Kg[8], Gg[8], cg[8];
      load8(bulK, g, i, j, k, Kn);
      load8(G, g, i, j, k, Gn);
      load8(gc, g, i, j, k, cn);
      gp_material(Kn, s, Kg);
      gp_material(Gn, s, Gg);
      gp_material(cn, s, cg);
      double gx[3][4], gy[3][4], gz[3][4];
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        double un[8];
        load8(u + m * g.n, g, i, j, k, un);
        sf_forward(un, s, gx[m], gy[m], gz[m], (double*)nullptr);
      }
      double tmp = 0.0;
#pragma unroll
      for (int gp = 0; gp < 8; ++gp) {
        Strain e8 = strain_at(gx, gy, gz, gp & 1, (gp >> 1) & 1, gp >> 2);
        e8.xx *= uprop; e8.yy *= uprop; e8.zz *= uprop; e8.xy *= uprop; e8.xz *= uprop; e8.yz *= uprop;
        tmp += phi_pos(Kg[gp], Gg[gp], e8) - 0.5 * cg[gp] / lc;
      }
      const double Ht = 0.125 * tmp;
      const long long e = nidx(g, i, j, k);
      if (H[e] < Ht) H[e] = Ht;
    }
  }
}
int launch_strain_history(hpc_ctx* c, double lc, double uprop) {
  const int L = c->maxlevel;
  const LevelGeo& g = c->L[L];
  const LevelFields& F = c->F[L];
  if (g.nx < 2 || g.ny < 2 || g.nz < 2) return HPC_OK;
  long long rows = (long long)(g.ny - 1) * (g.nz - 1);
  int grid = (int)(rows < num_sms_v() * 8LL ? rows : num_sms_v() * 8LL);
  strain_history_kernel<<<grid, 128, 0, c->stream>>>(g, F.u, F.bulK, F.G, F.gc, F.H, lc, uprop);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// fd_h (phase_field_right_hand_side.cpp:14-47) as a gather: each node sums its elements in the
// reference's scatter order (elements ascending in (k, j, i)), each element term being the
// reference's sequential sum over Gauss points of wg*2*H_e*N(g, corner); plain IEEE products and
// sums without contraction, so the result equals the reference's bit for bit.
__constant__ double c_N[8][8];  // N(g, n) in the reference's Gauss-point and corner numbering

__global__ void fd_h_kernel(LevelGeo g, const double* H, double* fd) {
  // reference corner numbering from offsets (a,b,c): (0,0,0)0 (1,0,0)1 (1,1,0)2 (0,1,0)3 ...
  const int corner[8] = {0, 1, 3, 2, 4, 5, 7, 6};  // indexed by a + 2b + 4c
  const double w2 = __dmul_rn(g.wg, 2.0);
  FOR_NODES(g) {
    double acc = 0.0;
    for (int c = 1; c >= 0; --c)
      for (int b = 1; b >= 0; --b)
        for (int a = 1; a >= 0; --a) {
          const int ex = i - a, ey = j - b, ez = kz - c;
          if (ex < 0 || ey < 0 || ez < 0 || ex > g.nx - 2 || ey > g.ny - 2 || ez > g.nz - 2) continue;
          const double h = H[nidx(g, ex, ey, ez)];
          const int tf = corner[a + 2 * b + 4 * c];
          const double wh = __dmul_rn(w2, h);
          double v = 0.0;
#pragma unroll
          for (int gp = 0; gp < 8; ++gp) v = __dadd_rn(v, __dmul_rn(wh, c_N[gp][tf]));
          acc = __dadd_rn(acc, v);
        }
    fd[nidx(g, i, j, kz)] = acc;
  }
}
int upload_shape_table(const double* N64) {
  cudaError_t e = cudaMemcpyToSymbol(c_N, N64, sizeof(double) * 64);
  return e == cudaSuccess ? HPC_OK : cuda_fail(e, "cudaMemcpyToSymbol(N)");
}
int launch_fd_h(hpc_ctx* c, int level) {
  const LevelGeo& g = c->L[level];
  fd_h_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(g, c->F[level].H, c->F[level].fd);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// delta_d_max and d_max (phase_field_max_search.cpp:17-53), fused with d_old = d.
__global__ void dmax_kernel(LevelGeo g, const double* d, double* dold, int copy, RedTarget red) {
  double dd = 0.0, dm = 0.0;
  FOR_NODES(g) {
    const long long n = nidx(g, i, j, kz);
    const double v = d[n];
    if (owned_plane(g, kz)) {
      dd = fmax(dd, v - dold[n]);
      dm = fmax(dm, v);
    }
    if (copy) dold[n] = v;
  }
  double r[2] = {dd, dm};
  grid_reduce<2, RED_MAX>(r, red);
}
int launch_dmax(hpc_ctx* c, int slot_dd, int slot_dmax, bool copy_old) {
  const int L = c->maxlevel;
  const LevelGeo& g = c->L[L];
  dmax_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(g, c->F[L].d, c->d_old, copy_old ? 1 : 0,
                                                         make_red(c, slot_dd, slot_dmax, -1, RED_MAX));
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// U_e (strain_history.cpp:86-131): min over elements and Gauss points of sqrt(phi_c / W).
__global__ void ue_kernel(LevelGeo g, const double* u, const double* bulK, const double* G, const double* gc,
                          double lc, RedTarget red) {
  const SF s = make_sf(g);
  double mn = 1e10;
  for (long long row = blockIdx.x; row < (long long)(g.ny - 1) * (g.nz - 1); row += gridDim.x) {
    const int j = (int)(row % (g.ny - 1)), k = (int)(row / (g.ny - 1));
    for (int i = threadIdx.x; i < g.nx - 1; i += blockDim.x) {
      double Kn[8], Gn[8], cn[8], Kg[8], Gg[8], cg[8];
      load8(bulK, g, i, j, k, Kn);
      load8(G, g, i, j, k, Gn);
      load8(gc, g, i, j, k, cn);
      gp_material(Kn, s, Kg);
      gp_material(Gn, s, Gg);
      gp_material(cn, s, cg);
      double gx[3][4], gy[3][4], gz[3][4];
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        double un[8];
        load8(u + m * g.n, g, i, j, k, un);
        sf_forward(un, s, gx[m], gy[m], gz[m], (double*)nullptr);
      }
#pragma unroll
      for (int gp = 0; gp < 8; ++gp) {
        const Strain e8 = strain_at(gx, gy, gz, gp & 1, (gp >> 1) & 1, gp >> 2);
        const double tr = e8.xx + e8.yy + e8.zz;
        const double K = Kg[gp], Gm = Gg[gp];
        // W = 1/2 sigma:eps with sigma = K tr I + 2G dev(eps)
        const double third = tr / 3.0;
        const double sxx = K * tr + 2.0 * Gm * (e8.xx - third);
        const double syy = K * tr + 2.0 * Gm * (e8.yy - third);
        const double szz = K * tr + 2.0 * Gm * (e8.zz - third);
        const double W0 = 0.5 * (sxx * e8.xx + syy * e8.yy + szz * e8.zz) +
                          0.5 * 2.0 * (2.0 * Gm) * (e8.xy * e8.xy + e8.xz * e8.xz + e8.yz * e8.yz);
        const double phic = 0.5 * cg[gp] / lc;
        const double ut = sqrt(phic / W0);
        if (ut < mn) mn = ut;
      }
    }
  }
  double r[1] = {mn};
  grid_reduce<1, RED_MIN>(r, red);
}
int launch_ue(hpc_ctx* c, double lc, int slot) {
  const int L = c->maxlevel;
  const LevelGeo& g = c->L[L];
  const LevelFields& F = c->F[L];
  long long rows = (long long)(g.ny - 1) * (g.nz - 1);
  int grid = (int)(rows < num_sms_v() * 8LL ? rows : num_sms_v() * 8LL);
  if (grid <= 0) grid = 1;
  ue_kernel<<<grid, 128, 0, c->stream>>>(g, F.u, F.bulK, F.G, F.gc, lc, make_red(c, slot, -1, -1, RED_MIN));
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// externe_force_sum (mechanical_right_hnd.cpp:40-59): sum of fu_z over the top node plane.
__global__ void top_sum_kernel(LevelGeo g, const double* fz, RedTarget red) {
  double s = 0.0;
  const int k = g.nz - 1;  // a slab rank below the top holds a ghost copy there: it adds nothing
  if (owned_plane(g, k))
    for (long long j = blockIdx.x; j < g.ny; j += gridDim.x)
      for (int i = threadIdx.x; i < g.nx; i += blockDim.x) s += fz[nidx(g, i, (int)j, k)];
  double r[1] = {s};
  grid_reduce<1>(r, red);
}
int launch_top_sum(hpc_ctx* c, int slot) {
  const int L = c->maxlevel;
  const LevelGeo& g = c->L[L];
  int grid = g.ny < num_sms_v() * 4 ? g.ny : num_sms_v() * 4;
  top_sum_kernel<<<grid, kRowThreads, 0, c->stream>>>(g, c->F[L].fu + 2 * g.n, make_red(c, slot, -1, -1));
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// initial_crack (strain_history.cpp:30-70); per-axis predicates come from the host, computed with
// the reference's coordinate arithmetic.
__global__ void crack_kernel(LevelGeo g, const uint8_t* fx, const uint8_t* fy, const uint8_t* fz, double* H,
                             double Hc) {
  FOR_NODES(g) {
    if (!fz[kz]) continue;
    if (!(fy[j] && fx[i])) H[nidx(g, i, j, kz)] = Hc;  // y != yb || x != xb
  }
}
int launch_crack(hpc_ctx* c, int level, const uint8_t* fx, const uint8_t* fy, const uint8_t* fz, double Hc) {
  crack_kernel<<<row_grid(c->L[level]), kRowThreads, 0, c->stream>>>(c->L[level], fx, fy, fz, c->F[level].H, Hc);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// image_MP (image_input.cpp:120-142): gray level -> (E, nu, Gc) with the reference's integer-division
// interpolation weight, E scaled by the voxel size, K = E/(3(1-2nu)), G = E/(2(1+nu)).
__global__ void image_material_kernel(LevelGeo g, const uint8_t* img, int vnx, int vny, int rx, int ry, int rz,
                                      int ngray, const int* gray, const double* E, const double* nu,
                                      const double* gcv, double voxel, double* bulK, double* G, double* gc,
                                      int* err) {
  FOR_NODES(g) {
    const long long vx = (long long)rx + i + (long long)vnx * (ry + j) + (long long)vnx * vny * (rz + g.zb + kz);
    const int gl = img[vx];
    int p = -1;
    for (int q = 0; q < ngray - 1; ++q)
      if (gl >= gray[q] && gl <= gray[q + 1]) { p = q; break; }
    const long long n = nidx(g, i, j, kz);
    if (p < 0 || gray[p + 1] == gray[p]) {
      atomicExch(err, 1);
      bulK[n] = G[n] = gc[n] = 0.0;
      continue;
    }
    const int w = (gl - gray[p]) / (gray[p + 1] - gray[p]);
    double Ev = __dadd_rn(E[p], __dmul_rn((double)w, __dsub_rn(E[p + 1], E[p])));
    const double nv = __dadd_rn(nu[p], __dmul_rn((double)w, __dsub_rn(nu[p + 1], nu[p])));
    gc[n] = __dadd_rn(gcv[p], __dmul_rn((double)w, __dsub_rn(gcv[p + 1], gcv[p])));
    Ev = __dmul_rn(voxel, Ev);
    bulK[n] = __dmul_rn(__ddiv_rn(1.0, __dmul_rn(3.0, __dsub_rn(1.0, __dmul_rn(2.0, nv)))), Ev);
    G[n] = __dmul_rn(__ddiv_rn(1.0, __dmul_rn(2.0, __dadd_rn(1.0, nv))), Ev);
  }
}
int launch_image_material(hpc_ctx* c, const uint8_t* dimage, const int* voxel_n, int ngray, const int* dgray,
                          const double* dE, const double* dnu, const double* dgc, double voxel_size) {
  const int L = c->maxlevel;
  const LevelGeo& g = c->L[L];
  const LevelFields& F = c->F[L];
  int* derr = reinterpret_cast<int*>(c->counter + 1);
  HPC_CUDA(cudaMemsetAsync(derr, 0, sizeof(int), c->stream));
  image_material_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(
      g, dimage, voxel_n[0], voxel_n[1], c->geo.roi_start[0], c->geo.roi_start[1], c->geo.roi_start[2], ngray, dgray,
      dE, dnu, dgc, voxel_size, F.bulK, F.G, F.gc, derr);
  HPC_CHECK_LAUNCH(c);
  int herr = 0;
  HPC_CUDA(cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  if (herr) {
    set_error("gray level outside the material table (findPosition returned -1, csv_reader.cpp:65-73)");
    return HPC_ERR_INPUT;
  }
  return HPC_OK;
}

// Count of zero entries of a diagonal on valid nodes (the reference throws on them, grid.h:182-190).
__global__ void zero_count_kernel(LevelGeo g, int ncomp, const double* v, RedTarget red) {
  double cnt = 0.0;
  FOR_NODES(g) {
    if (!owned_plane(g, kz)) continue;
    const long long n = nidx(g, i, j, kz);
    for (int m = 0; m < ncomp; ++m) cnt += (v[n + m * g.n] == 0.0) ? 1.0 : 0.0;
  }
  double r[1] = {cnt};
  grid_reduce<1>(r, red);
}
int launch_zero_count(hpc_ctx* c, int level, int ncomp, const double* v, int slot) {
  const LevelGeo& g = c->L[level];
  zero_count_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(g, ncomp, v, make_red(c, slot, -1, -1));
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

}  // namespace hpc

// ---------------------------------------------------------------------------------------------
// Precision form: the V-cycle's vector kernels on the FP32 mirror of the levels (homogeneous
// Dirichlet values: the cycle solves for a correction), and FP64 <-> FP32 conversions.
// ---------------------------------------------------------------------------------------------
namespace hpc {
namespace {
template <typename S, typename D>
__global__ void convert_kernel(const S* src, D* dst, long long n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    dst[q] = (D)src[q];
}
int flat_grid(long long n) {
  const long long blocks = (n + kRowThreads - 1) / kRowThreads, cap = (long long)num_sms_v() * 8;
  return (int)(blocks < cap ? blocks : cap);
}
}  // namespace

int launch_to_f32(hpc_ctx* c, const double* src, float* dst, long long n) {
  convert_kernel<<<flat_grid(n), kRowThreads, 0, c->stream>>>(src, dst, n);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}
// Dense x-fastest host layout -> the level's pitched layout (the upload's second half: one
// contiguous host-to-device copy into `dense`, then this kernel on the device).
__global__ void unpack_kernel(LevelGeo g, const double* dense, double* dst) {
  const long long total = (long long)g.nx * g.ny * g.nz;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx);
    const long long r = q / g.nx;
    const int j = (int)(r % g.ny), k = (int)(r / g.ny);
    dst[nidx(g, i, j, k)] = dense[q];
  }
}

int launch_unpack(hpc_ctx* c, int level, const double* dense, double* dst) {
  const LevelGeo& g = c->L[level];
  unpack_kernel<<<flat_grid((long long)g.nx * g.ny * g.nz), kRowThreads, 0, c->stream>>>(g, dense, dst);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

int launch_to_f64(hpc_ctx* c, const float* src, double* dst, long long n) {
  convert_kernel<<<flat_grid(n), kRowThreads, 0, c->stream>>>(src, dst, n);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

int launch_mech_update_f32(hpc_ctx* c, int level, int s_num, int s_den, int s_rz_next, int s_rn) {
  const LevelGeo& g = c->L[level];
  const LevelF32& F = c->F32[level];
  const long long pairs = (long long)(g.px / 2) * g.ny * g.nz;
  const int grid = (int)std::min<long long>((pairs + kRowThreads - 1) / kRowThreads, (long long)num_sms_v() * 8);
  if (c->slab)
    mech_update_kernel<float, true><<<grid, kRowThreads, 0, c->stream>>>(g, F.u, F.ru, F.p, F.w, F.invM, s_num, s_den,
                                                                       make_red(c, s_rz_next, s_rn, -1));
  else
    mech_update_kernel<float, false><<<grid, kRowThreads, 0, c->stream>>>(g, F.u, F.ru, F.p, F.w, F.invM, s_num,
                                                                        s_den, make_red(c, s_rz_next, s_rn, -1));
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}
int launch_dir_update_f32(hpc_ctx* c, int level, bool first, int s_rz, int s_rz_prev) {
  const LevelGeo& g = c->L[level];
  const LevelF32& F = c->F32[level];
  dir_update_kernel<float><<<row_grid(g), kRowThreads, 0, c->stream>>>(g, 3, F.ru, F.invM, F.p, first ? 1 : 0,
                                                                       c->scal, s_rz, s_rz_prev);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, level, F.p, 3, sizeof(float));
  return HPC_OK;
}
int launch_bc_zero_f32(hpc_ctx* c, int level, float* v) {
  const LevelGeo& g = c->L[level];
  bc_kernel<float><<<row_grid(g), kRowThreads, 0, c->stream>>>(g, v, nullptr, 2, 0.0f);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}
int launch_inject_u_f32(hpc_ctx* c, int lf) {
  inject_u_kernel<float><<<row_grid(c->L[lf - 1]), kRowThreads, 0, c->stream>>>(
      c->L[lf - 1], c->L[lf], c->F32[lf].u, c->F32[lf - 1].u, c->F32[lf - 1].uold, 0.0f);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, lf - 1, c->F32[lf - 1].u, 3, sizeof(float));
  HPC_SLAB_HALO(c, lf - 1, c->F32[lf - 1].uold, 3, sizeof(float));
  return HPC_OK;
}
int launch_prolong_f32(hpc_ctx* c, int lf) {
  prolong_kernel<float><<<row_grid(c->L[lf]), kRowThreads, 0, c->stream>>>(
      c->L[lf - 1], c->L[lf], c->F32[lf - 1].u, c->F32[lf - 1].uold, c->F32[lf].u, 3, 1, 0.0f);
  HPC_CHECK_LAUNCH(c);
  HPC_SLAB_HALO(c, lf, c->F32[lf].u, 3, sizeof(float));
  return HPC_OK;
}
}  // namespace hpc

namespace hpc {
// The residual of the correction problem when its unknown is still zero: r = f with Dirichlet rows
// zero, (r, M^-1 r) into a slot - the first residual of the precision form's finest pre-smoother,
// without an operator apply.
__global__ void residual_zero_f32_kernel(LevelGeo g, const float* f, const float* invM, float* r, RedTarget red) {
  double rz = 0.0;
  FOR_NODES(g) {
    const long long n = nidx(g, i, j, kz);
    bool fix[3] = {false, false, false};
    if (g.bz[kz]) {
      const BcFlags bc = bc_flags(g, i, j, kz);
      fix[0] = bc.c0;
      fix[1] = bc.c1;
      fix[2] = bc.c2;
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const long long o = n + (long long)m * g.n;
      const float rv = fix[m] ? 0.f : f[o];
      r[o] = rv;
      const double s1 = fma((double)rv, (double)(rv * invM[o]), rz);
      rz = owned_plane(g, kz) ? s1 : rz;
    }
  }
  double v[1] = {rz};
  grid_reduce<1>(v, red);
}

int launch_residual_zero_f32(hpc_ctx* c, int level, int s_rz) {
  const LevelGeo& g = c->L[level];
  const LevelF32& F = c->F32[level];
  residual_zero_f32_kernel<<<row_grid(g), kRowThreads, 0, c->stream>>>(g, F.fu, F.invM, F.ru,
                                                                       make_red(c, s_rz, -1, -1));
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}
}  // namespace hpc
