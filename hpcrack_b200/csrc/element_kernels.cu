// Element-operator kernels: mechanical K(d) u and diag K(d), phase-field A_d x and diag A_d, with
// fused epilogues (residual, PCG direction update, FAS right-hand side, reactions).
//
// Tiling ("warp strip"): each warp owns a strip of 32 node columns in x (31 elements, 30 output nodes),
// WY element rows in y (WY-1 output node rows) and CZ output node planes in z, and marches in z.
// Per element row a lane computes one element; the x-neighbour contributions are combined with
// one shuffle, y-neighbours through registers (the previous row's upper-face sums) and
// z-neighbours through a per-warp shared-memory carry of the previous layer's upper faces.  Every
// node is written once, by the warp whose output range owns it, with a fixed summation order:
// no atomics, no block-wide barriers in the march, deterministic results.  Warps stride over the
// strip list (persistent grid).
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "internal.h"

namespace hpc {

constexpr int kWarps = 4;    // warps per block
constexpr int kWY = 8;       // element rows per strip (kWY - 1 output node rows)
constexpr int kCZ = 16;      // output planes per strip
constexpr int kOX = 30;      // output nodes per strip in x (lanes 1..30)

struct StripGeo {
  int tx, ty, tz;            // strips per axis
  long long nstrips;
};

__host__ __device__ inline StripGeo strip_geo(const LevelGeo& g) {
  StripGeo s;
  s.tx = (g.nx + kOX - 1) / kOX;
  s.ty = (g.ny + kWY - 2) / (kWY - 1);
  s.tz = (g.nz + kCZ - 1) / kCZ;
  s.nstrips = (long long)s.tx * s.ty * s.tz;
  return s;
}

// ------------------------------------------------------------------------------------------
// mechanical
// ------------------------------------------------------------------------------------------
struct MechK {
  LevelGeo g;
  LevelGeo gf;  // fine level (FAS)
  StripGeo sg;
  int finest, epi, diag, set_fnorm, first;
  const double* src;
  double* out;
  const double *bulK, *G, *d, *Ke, *Ge;
  const int8_t* choice;
  double small_k;
  double* fu;
  const double* invM;
  const double* r;
  double* p_new;
  const double* rf;
  int s_rz, s_rz_prev;
  RedTarget red;
};

// Node values a lane needs for its elements: displacement (or the PCG direction being formed)
// and, on the finest level, the nodal moduli and phase field.
struct MechNode {
  double u[3];
  double K, G, d;
};

template <bool FINEST, int EPI>
__device__ __forceinline__ MechNode mech_load(const MechK& k, int x, int y, int z, double beta) {
  MechNode v;
  const bool ok = x >= 0 && x < k.g.nx && y >= 0 && y < k.g.ny && z >= 0 && z < k.g.nz;
  const long long n = ok ? (long long)x + (long long)y * k.g.px + (long long)z * k.g.plane : 0;
  if (EPI == EPI_PCG) {
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      double pv = 0.0;
      if (ok) {
        const long long o = n + (long long)m * k.g.n;
        const double zv = k.r[o] * k.invM[o];
        pv = k.first ? zv : fma(beta, k.src[o], zv);
      }
      v.u[m] = pv;
    }
  } else {
#pragma unroll
    for (int m = 0; m < 3; ++m) v.u[m] = ok ? k.src[n + (long long)m * k.g.n] : 0.0;
  }
  if (FINEST) {
    v.K = ok ? k.bulK[n] : 0.0;
    v.G = ok ? k.G[n] : 0.0;
    v.d = ok ? k.d[n] : 0.0;
  } else {
    v.K = v.G = v.d = 0.0;
  }
  return v;
}

__device__ __forceinline__ double shfl_down1(double v) { return __shfl_down_sync(kFull, v, 1); }

// Per-Gauss-point moduli times wg (MP_all_GAUSS_Point, mechanical_pcg.cpp:26-61).
template <bool FINEST>
__device__ __forceinline__ void mech_moduli(const MechK& k, const MechNode (&nd)[8], long long e, const SF& s,
                                            double (&Kw)[8], double (&Gw)[8]) {
  const double wg = k.g.wg;
  if (FINEST) {
    double v[8], Kg[8], Gg[8], dg[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) v[n] = nd[n].K;
    gp_material(v, s, Kg);
#pragma unroll
    for (int n = 0; n < 8; ++n) v[n] = nd[n].G;
    gp_material(v, s, Gg);
    const int ch = k.choice[e];
    if (ch == 2) {
#pragma unroll
      for (int g = 0; g < 8; ++g) { Kw[g] = Kg[g] * wg; Gw[g] = Gg[g] * wg; }
    } else {
#pragma unroll
      for (int n = 0; n < 8; ++n) v[n] = nd[n].d;
      gp_material(v, s, dg);
      const double sk = k.small_k;
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        const double dd = fmin(fmax(dg[g], 0.0), 1.0);  // K_G_d_g clamp (material_gauss_point.cpp:51-54)
        const double om = 1.0 - dd;
        const double gd = fma((1.0 - sk) * om, om, sk);
        Kw[g] = (ch == 0 ? gd * Kg[g] : Kg[g]) * wg;
        Gw[g] = (gd * Gg[g]) * wg;
      }
    }
  } else {
    const double K = k.Ke[e] * wg, G = k.Ge[e] * wg;
#pragma unroll
    for (int g = 0; g < 8; ++g) { Kw[g] = K; Gw[g] = G; }
  }
}

template <bool FINEST, int EPI, bool DIAG>
__global__ void __launch_bounds__(kWarps * 32) mech_kernel(MechK k) {
  extern __shared__ double zc_all[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* zc = zc_all + (size_t)wib * (kWY - 1) * 3 * 32;  // [row][comp][lane]
  const SF s = make_sf(k.g);
  const double beta =
      (EPI == EPI_PCG && !k.first) ? k.red.scal[k.s_rz] / k.red.scal[k.s_rz_prev] : 0.0;
  double red0 = 0.0, red1 = 0.0, red2 = 0.0;
  const long long nwarps_total = (long long)gridDim.x * kWarps;

  for (long long strip = (long long)blockIdx.x * kWarps + wib; strip < k.sg.nstrips; strip += nwarps_total) {
    const int sx = (int)(strip % k.sg.tx);
    const long long rest = strip / k.sg.tx;
    const int sy = (int)(rest % k.sg.ty);
    const int sz = (int)(rest / k.sg.ty);
    const int x0 = sx * kOX, y0 = sy * (kWY - 1), z0 = sz * kCZ;
    const int x = x0 - 1 + lane;
    const int zend = min(z0 + kCZ - 1, k.g.nz - 1);
    for (int kk = z0 - 1; kk <= zend; ++kk) {
      double yp[2][3];  // previous element row's upper-y-face sums, [c][m]
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int m = 0; m < 3; ++m) yp[c][m] = 0.0;
      for (int rr = 0; rr < kWY; ++rr) {
        const int ey = y0 - 1 + rr;
        // ---- gather the element's 8 nodes: own column x, x+1 from the next lane
        MechNode nd[8];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int b = 0; b < 2; ++b) nd[2 * b + 4 * c] = mech_load<FINEST, EPI>(k, x, ey + b, kk + c, beta);
        MechNode own00 = nd[0];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            MechNode& o = nd[2 * b + 4 * c];
            MechNode& t = nd[1 + 2 * b + 4 * c];
#pragma unroll
            for (int m = 0; m < 3; ++m) t.u[m] = shfl_down1(o.u[m]);
            if (FINEST) { t.K = shfl_down1(o.K); t.G = shfl_down1(o.G); t.d = shfl_down1(o.d); }
          }
        // ---- element contribution (lane 31 has no right neighbour: its element belongs to the next strip)
        double f[3][8];
        const bool valid = lane < 31 && x >= 0 && x <= k.g.nx - 2 && ey >= 0 && ey <= k.g.ny - 2 && kk >= 0 &&
                           kk <= k.g.nz - 2;
        if (valid) {
          const long long e = (long long)x + (long long)ey * k.g.px + (long long)kk * k.g.plane;
          double Kw[8], Gw[8];
          mech_moduli<FINEST>(k, nd, e, s, Kw, Gw);
          if (DIAG) {
            mech_element_diag(Kw, Gw, s, f);
          } else {
            double u[3][8];
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
              for (int n = 0; n < 8; ++n) u[m][n] = nd[n].u[m];
            mech_element(u, Kw, Gw, s, f);
          }
        } else {
#pragma unroll
          for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int n = 0; n < 8; ++n) f[m][n] = 0.0;
        }
        // ---- combine x-neighbours: node x gets own a=0 corners + left lane's a=1 corners
        double X[2][2][3];  // [b][c][m]
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int m = 0; m < 3; ++m) {
              const double left = __shfl_up_sync(kFull, f[m][1 + 2 * b + 4 * c], 1);
              X[b][c][m] = f[m][2 * b + 4 * c] + (lane > 0 ? left : 0.0);
            }
        if (rr >= 1) {
          const int orow = rr - 1;
          double tot[3];
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            double* zp = zc + (orow * 3 + m) * 32 + lane;
            tot[m] = *zp + yp[0][m] + X[0][0][m];
            *zp = yp[1][m] + X[0][1][m];
          }
          if (kk >= z0 && lane >= 1 && lane <= 30 && x < k.g.nx && ey < k.g.ny) {
            const long long n = (long long)x + (long long)ey * k.g.px + (long long)kk * k.g.plane;
            const long long N = k.g.n;
            if (EPI == EPI_PLAIN) {
#pragma unroll
              for (int m = 0; m < 3; ++m) k.out[n + m * N] = tot[m];
            } else if (EPI == EPI_RESIDUAL) {
              const BcFlags bc = bc_flags(k.g, x, ey, kk);
              const bool fix[3] = {bc.c0, bc.c1, bc.c2};
#pragma unroll
              for (int m = 0; m < 3; ++m) {
                double fv = k.fu[n + m * N];
                if (k.set_fnorm && fix[m]) {
                  fv = tot[m];
                  k.fu[n + m * N] = fv;
                }
                red0 = fma(fv, fv, red0);
                double rv = fix[m] ? 0.0 : fv - tot[m];
                k.out[n + m * N] = rv;
                if (k.invM) red1 = fma(rv, rv * k.invM[n + m * N], red1);
                red2 = fma(rv, rv, red2);
              }
            } else if (EPI == EPI_PCG) {
#pragma unroll
              for (int m = 0; m < 3; ++m) {
                k.out[n + m * N] = tot[m];
                k.p_new[n + m * N] = own00.u[m];
                red0 = fma(own00.u[m], tot[m], red0);
              }
            } else if (EPI == EPI_FAS) {
              // coarsen_f_standard_routine (multigrid_intergrid.cpp:124-342) fused with the coarse apply
              const int fx = 2 * x, fy = 2 * ey, fz = 2 * kk;
              const int Xl = k.gf.nx - 2, Yl = k.gf.ny - 2, Zl = k.gf.nz - 2;
#pragma unroll
              for (int m = 0; m < 3; ++m) {
                const double* rf = k.rf + (long long)m * k.gf.n;
                auto R = [&](int a, int b, int c) -> double {
                  return rf[(long long)a + (long long)b * k.gf.px + (long long)c * k.gf.plane];
                };
                const bool xm = fx < 1, xp = fx > Xl, ym = fy < 1, yq = fy > Yl, zm = fz < 1, zq = fz > Zl;
                const double r11 = (xm || ym || zm) ? 0.0 : R(fx - 1, fy - 1, fz - 1);
                const double r12 = (xm || ym || zq) ? 0.0 : R(fx - 1, fy - 1, fz + 1);
                const double r13 = (xm || yq || zm) ? 0.0 : R(fx - 1, fy + 1, fz - 1);
                const double r14 = (xm || yq || zq) ? 0.0 : R(fx - 1, fy + 1, fz + 1);
                const double r15 = (xp || ym || zm) ? 0.0 : R(fx + 1, fy - 1, fz - 1);
                const double r16 = (xp || ym || zq) ? 0.0 : R(fx + 1, fy - 1, fz + 1);
                const double r17 = (xp || yq || zm) ? 0.0 : R(fx + 1, fy + 1, fz - 1);
                const double r18 = (xp || yq || zq) ? 0.0 : R(fx + 1, fy + 1, fz + 1);
                const double r21 = (xm || ym) ? 0.0 : R(fx - 1, fy - 1, fz);
                const double r22 = (xm || yq) ? 0.0 : R(fx - 1, fy + 1, fz);
                const double r23 = (xp || ym) ? 0.0 : R(fx + 1, fy - 1, fz);
                const double r24 = (xp || yq) ? 0.0 : R(fx + 1, fy + 1, fz);
                const double r25 = (xm || zm) ? 0.0 : R(fx - 1, fy, fz - 1);
                const double r26 = (xm || zq) ? 0.0 : R(fx - 1, fy, fz + 1);
                const double r27 = (xp || zm) ? 0.0 : R(fx + 1, fy, fz - 1);
                const double r28 = (xp || zq) ? 0.0 : R(fx + 1, fy, fz + 1);
                const double r29 = (ym || zm) ? 0.0 : R(fx, fy - 1, fz - 1);
                const double r210 = (ym || zq) ? 0.0 : R(fx, fy - 1, fz + 1);
                const double r211 = (yq || zm) ? 0.0 : R(fx, fy + 1, fz - 1);
                const double r212 = (yq || zq) ? 0.0 : R(fx, fy + 1, fz + 1);
                const double r41 = zm ? 0.0 : R(fx, fy, fz - 1);
                const double r42 = zq ? 0.0 : R(fx, fy, fz + 1);
                const double r43 = ym ? 0.0 : R(fx, fy - 1, fz);
                const double r44 = yq ? 0.0 : R(fx, fy + 1, fz);
                const double r45 = xm ? 0.0 : R(fx - 1, fy, fz);
                const double r46 = xp ? 0.0 : R(fx + 1, fy, fz);
                const double r8 = R(fx, fy, fz);
                const double s8 = r11 + r12 + r13 + r14 + r15 + r16 + r17 + r18;
                const double s12 = r21 + r22 + r23 + r24 + r25 + r26 + r27 + r28 + r29 + r210 + r211 + r212;
                const double s6 = r41 + r42 + r43 + r44 + r45 + r46;
                k.out[n + m * N] = tot[m] + 0.125 * (s8 + 2.0 * s12 + 4.0 * s6 + 8.0 * r8);
              }
            } else if (EPI == EPI_REACTION) {
              // Dirichlet_force_u (boundary_conditions.cpp:69-111)
              const BcFlags bc = bc_flags(k.g, x, ey, kk);
              if (bc.c0) k.out[n] = tot[0];
              if (bc.c1) k.out[n + N] = tot[1];
              if (bc.c2) k.out[n + 2 * N] = tot[2];
            }
          }
        }
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int m = 0; m < 3; ++m) yp[c][m] = X[1][c][m];
      }
    }
    __syncwarp();
  }
  if (EPI == EPI_RESIDUAL || EPI == EPI_PCG) {
    double v[3] = {red0, red1, red2};
    grid_reduce<3>(v, k.red);
  }
}

static int g_num_sms = 0;
static int num_sms() {
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

static size_t strip_smem() { return (size_t)kWarps * (kWY - 1) * 3 * 32 * sizeof(double); }

static int grid_for(const StripGeo& sg, int blocks_per_sm) {
  long long need = (sg.nstrips + kWarps - 1) / kWarps;
  long long cap = (long long)num_sms() * blocks_per_sm;
  return (int)(need < cap ? need : cap);
}

RedTarget make_red(hpc_ctx* c, int s0, int s1, int s2) {
  RedTarget t;
  t.partials = c->partials;
  t.counter = c->counter;
  t.scal = c->scal;
  t.slot[0] = s0;
  t.slot[1] = s1;
  t.slot[2] = s2;
  return t;
}

template <bool F, int E, bool D>
static int run_mech(hpc_ctx* c, const MechK& k) {
  const int grid = grid_for(k.sg, 3);
  if (grid <= 0) return HPC_OK;
  if ((size_t)grid * 3 > c->partials_cap) return cuda_fail(cudaErrorInvalidValue, "partials buffer");
  const int cls = (F && E == EPI_PCG && !D) ? HPC_KC_MECH_PCG_FINEST : HPC_KC_NONE;
  timing_begin(c, cls);
  mech_kernel<F, E, D><<<grid, kWarps * 32, strip_smem(), c->stream>>>(k);
  timing_end(c, cls);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

int launch_mech(hpc_ctx* c, const MechCall& m) {
  MechK k{};
  k.g = c->L[m.level];
  if (m.epi == EPI_FAS) k.gf = c->L[m.fine_level];
  k.sg = strip_geo(k.g);
  k.finest = m.finest;
  k.epi = m.epi;
  k.src = m.src;
  k.out = m.out;
  const LevelFields& F = c->F[m.level];
  k.bulK = F.bulK;
  k.G = F.G;
  k.d = F.d;
  k.Ke = F.Ke;
  k.Ge = F.Ge;
  k.choice = F.choice;
  k.small_k = m.small_k;
  k.fu = m.fu;
  k.set_fnorm = m.set_fnorm;
  k.invM = m.invM;
  k.r = m.r;
  k.p_new = m.p_new;
  k.first = m.first;
  k.s_rz = m.s_rz;
  k.s_rz_prev = m.s_rz_prev;
  k.rf = m.rf;
  k.red = make_red(c, m.s_out0, m.s_out1, m.s_out2);
  const bool f = m.finest;
  switch (m.epi) {
    case EPI_PLAIN: return f ? run_mech<true, EPI_PLAIN, false>(c, k) : run_mech<false, EPI_PLAIN, false>(c, k);
    case EPI_RESIDUAL:
      return f ? run_mech<true, EPI_RESIDUAL, false>(c, k) : run_mech<false, EPI_RESIDUAL, false>(c, k);
    case EPI_PCG: return f ? run_mech<true, EPI_PCG, false>(c, k) : run_mech<false, EPI_PCG, false>(c, k);
    case EPI_FAS: return run_mech<false, EPI_FAS, false>(c, k);
    case EPI_REACTION:
      return f ? run_mech<true, EPI_REACTION, false>(c, k) : run_mech<false, EPI_REACTION, false>(c, k);
  }
  return HPC_ERR_ARG;
}

int launch_mech_diag(hpc_ctx* c, int level, bool finest, double small_k, double* out) {
  MechCall m{};
  m.level = level;
  MechK k{};
  k.g = c->L[level];
  k.sg = strip_geo(k.g);
  const LevelFields& F = c->F[level];
  k.bulK = F.bulK;
  k.G = F.G;
  k.d = F.d;
  k.Ke = F.Ke;
  k.Ge = F.Ge;
  k.choice = F.choice;
  k.small_k = small_k;
  k.src = F.u;  // unused by the diagonal
  k.out = out;
  k.red = make_red(c, -1, -1, -1);
  return finest ? run_mech<true, EPI_PLAIN, true>(c, k) : run_mech<false, EPI_PLAIN, true>(c, k);
}

// ------------------------------------------------------------------------------------------
// phase field
// ------------------------------------------------------------------------------------------
struct PfK {
  LevelGeo g, gf;
  StripGeo sg;
  int epi, first;
  const double* src;
  double* out;
  const double *gc, *H;
  double lc;
  const double* fd;
  const double* invM;
  const double* r;
  double* p_new;
  const double* rf;
  int s_rz, s_rz_prev;
  RedTarget red;
};

struct PfNode {
  double x, gc;
};

template <int EPI>
__device__ __forceinline__ PfNode pf_load(const PfK& k, int x, int y, int z, double beta) {
  PfNode v;
  const bool ok = x >= 0 && x < k.g.nx && y >= 0 && y < k.g.ny && z >= 0 && z < k.g.nz;
  const long long n = ok ? (long long)x + (long long)y * k.g.px + (long long)z * k.g.plane : 0;
  if (EPI == EPI_PCG) {
    double pv = 0.0;
    if (ok) {
      const double zv = k.r[n] * k.invM[n];
      pv = k.first ? zv : fma(beta, k.src[n], zv);
    }
    v.x = pv;
  } else {
    v.x = ok ? k.src[n] : 0.0;
  }
  v.gc = ok ? k.gc[n] : 0.0;
  return v;
}

template <int EPI, bool DIAG>
__global__ void __launch_bounds__(kWarps * 32) pf_kernel(PfK k) {
  extern __shared__ double zc_all[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* zc = zc_all + (size_t)wib * (kWY - 1) * 32;  // [row][lane]
  const SF s = make_sf(k.g);
  const double beta = (EPI == EPI_PCG && !k.first) ? k.red.scal[k.s_rz] / k.red.scal[k.s_rz_prev] : 0.0;
  double red0 = 0.0, red1 = 0.0, red2 = 0.0;
  const long long nwarps_total = (long long)gridDim.x * kWarps;
  const double wg = k.g.wg, inv_lc = 1.0 / k.lc;

  for (long long strip = (long long)blockIdx.x * kWarps + wib; strip < k.sg.nstrips; strip += nwarps_total) {
    const int sx = (int)(strip % k.sg.tx);
    const long long rest = strip / k.sg.tx;
    const int sy = (int)(rest % k.sg.ty);
    const int sz = (int)(rest / k.sg.ty);
    const int x0 = sx * kOX, y0 = sy * (kWY - 1), z0 = sz * kCZ;
    const int x = x0 - 1 + lane;
    const int zend = min(z0 + kCZ - 1, k.g.nz - 1);
    for (int kk = z0 - 1; kk <= zend; ++kk) {
      double yp[2] = {0.0, 0.0};
      for (int rr = 0; rr < kWY; ++rr) {
        const int ey = y0 - 1 + rr;
        PfNode nd[8];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int b = 0; b < 2; ++b) nd[2 * b + 4 * c] = pf_load<EPI>(k, x, ey + b, kk + c, beta);
        const double own00 = nd[0].x;
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            nd[1 + 2 * b + 4 * c].x = shfl_down1(nd[2 * b + 4 * c].x);
            nd[1 + 2 * b + 4 * c].gc = shfl_down1(nd[2 * b + 4 * c].gc);
          }
        double f[8];
        const bool valid = lane < 31 && x >= 0 && x <= k.g.nx - 2 && ey >= 0 && ey <= k.g.ny - 2 && kk >= 0 &&
                           kk <= k.g.nz - 2;
        if (valid) {
          const long long e = (long long)x + (long long)ey * k.g.px + (long long)kk * k.g.plane;
          double gcn[8], gcg[8], aw[8], bw[8];
#pragma unroll
          for (int n = 0; n < 8; ++n) gcn[n] = nd[n].gc;
          gp_material(gcn, s, gcg);
          const double H2 = 2.0 * k.H[e];
#pragma unroll
          for (int g = 0; g < 8; ++g) {
            aw[g] = wg * fma(gcg[g], inv_lc, H2);
            bw[g] = wg * (gcg[g] * k.lc);
          }
          if (DIAG) {
            pf_element_diag(aw, bw, s, f);
          } else {
            double xv[8];
#pragma unroll
            for (int n = 0; n < 8; ++n) xv[n] = nd[n].x;
            pf_element(xv, aw, bw, s, f);
          }
        } else {
#pragma unroll
          for (int n = 0; n < 8; ++n) f[n] = 0.0;
        }
        double X[2][2];
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int b = 0; b < 2; ++b) {
            const double left = __shfl_up_sync(kFull, f[1 + 2 * b + 4 * c], 1);
            X[b][c] = f[2 * b + 4 * c] + (lane > 0 ? left : 0.0);
          }
        if (rr >= 1) {
          double* zp = zc + (rr - 1) * 32 + lane;
          const double tot = *zp + yp[0] + X[0][0];
          *zp = yp[1] + X[0][1];
          if (kk >= z0 && lane >= 1 && lane <= 30 && x < k.g.nx && ey < k.g.ny) {
            const long long n = (long long)x + (long long)ey * k.g.px + (long long)kk * k.g.plane;
            if (EPI == EPI_PLAIN) {
              k.out[n] = tot;
            } else if (EPI == EPI_RESIDUAL) {
              const double fv = k.fd[n];
              const double rv = fv - tot;
              k.out[n] = rv;
              red0 = fma(fv, fv, red0);
              red1 = fma(rv, rv, red1);
              if (k.invM) red2 = fma(rv, rv * k.invM[n], red2);
            } else if (EPI == EPI_PCG) {
              k.out[n] = tot;
              k.p_new[n] = own00;
              red0 = fma(own00, tot, red0);
            } else if (EPI == EPI_FAS) {
              const int fx = 2 * x, fy = 2 * ey, fz = 2 * kk;
              const int Xl = k.gf.nx - 2, Yl = k.gf.ny - 2, Zl = k.gf.nz - 2;
              const double* rf = k.rf;
              auto R = [&](int a, int b, int c2) -> double {
                return rf[(long long)a + (long long)b * k.gf.px + (long long)c2 * k.gf.plane];
              };
              const bool xm = fx < 1, xp = fx > Xl, ym = fy < 1, yq = fy > Yl, zm = fz < 1, zq = fz > Zl;
              const double r11 = (xm || ym || zm) ? 0.0 : R(fx - 1, fy - 1, fz - 1);
              const double r12 = (xm || ym || zq) ? 0.0 : R(fx - 1, fy - 1, fz + 1);
              const double r13 = (xm || yq || zm) ? 0.0 : R(fx - 1, fy + 1, fz - 1);
              const double r14 = (xm || yq || zq) ? 0.0 : R(fx - 1, fy + 1, fz + 1);
              const double r15 = (xp || ym || zm) ? 0.0 : R(fx + 1, fy - 1, fz - 1);
              const double r16 = (xp || ym || zq) ? 0.0 : R(fx + 1, fy - 1, fz + 1);
              const double r17 = (xp || yq || zm) ? 0.0 : R(fx + 1, fy + 1, fz - 1);
              const double r18 = (xp || yq || zq) ? 0.0 : R(fx + 1, fy + 1, fz + 1);
              const double r21 = (xm || ym) ? 0.0 : R(fx - 1, fy - 1, fz);
              const double r22 = (xm || yq) ? 0.0 : R(fx - 1, fy + 1, fz);
              const double r23 = (xp || ym) ? 0.0 : R(fx + 1, fy - 1, fz);
              const double r24 = (xp || yq) ? 0.0 : R(fx + 1, fy + 1, fz);
              const double r25 = (xm || zm) ? 0.0 : R(fx - 1, fy, fz - 1);
              const double r26 = (xm || zq) ? 0.0 : R(fx - 1, fy, fz + 1);
              const double r27 = (xp || zm) ? 0.0 : R(fx + 1, fy, fz - 1);
              const double r28 = (xp || zq) ? 0.0 : R(fx + 1, fy, fz + 1);
              const double r29 = (ym || zm) ? 0.0 : R(fx, fy - 1, fz - 1);
              const double r210 = (ym || zq) ? 0.0 : R(fx, fy - 1, fz + 1);
              const double r211 = (yq || zm) ? 0.0 : R(fx, fy + 1, fz - 1);
              const double r212 = (yq || zq) ? 0.0 : R(fx, fy + 1, fz + 1);
              const double r41 = zm ? 0.0 : R(fx, fy, fz - 1);
              const double r42 = zq ? 0.0 : R(fx, fy, fz + 1);
              const double r43 = ym ? 0.0 : R(fx, fy - 1, fz);
              const double r44 = yq ? 0.0 : R(fx, fy + 1, fz);
              const double r45 = xm ? 0.0 : R(fx - 1, fy, fz);
              const double r46 = xp ? 0.0 : R(fx + 1, fy, fz);
              const double r8 = R(fx, fy, fz);
              const double s8 = r11 + r12 + r13 + r14 + r15 + r16 + r17 + r18;
              const double s12 = r21 + r22 + r23 + r24 + r25 + r26 + r27 + r28 + r29 + r210 + r211 + r212;
              const double s6 = r41 + r42 + r43 + r44 + r45 + r46;
              k.out[n] = tot + 0.125 * (s8 + 2.0 * s12 + 4.0 * s6 + 8.0 * r8);
            }
          }
        }
        yp[0] = X[1][0];
        yp[1] = X[1][1];
      }
    }
    __syncwarp();
  }
  if (EPI == EPI_RESIDUAL || EPI == EPI_PCG) {
    double v[3] = {red0, red1, red2};
    grid_reduce<3>(v, k.red);
  }
}

static size_t strip_smem_pf() { return (size_t)kWarps * (kWY - 1) * 32 * sizeof(double); }

template <int E, bool D>
static int run_pf(hpc_ctx* c, const PfK& k, bool finest) {
  const int grid = grid_for(k.sg, 4);
  if (grid <= 0) return HPC_OK;
  if ((size_t)grid * 3 > c->partials_cap) return cuda_fail(cudaErrorInvalidValue, "partials buffer");
  const int cls = (finest && E == EPI_PCG && !D) ? HPC_KC_PF_PCG_FINEST : HPC_KC_NONE;
  timing_begin(c, cls);
  pf_kernel<E, D><<<grid, kWarps * 32, strip_smem_pf(), c->stream>>>(k);
  timing_end(c, cls);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

int launch_pf(hpc_ctx* c, const PfCall& p) {
  PfK k{};
  k.g = c->L[p.level];
  if (p.epi == EPI_FAS) k.gf = c->L[p.fine_level];
  k.sg = strip_geo(k.g);
  k.epi = p.epi;
  k.first = p.first;
  k.src = p.src;
  k.out = p.out;
  k.gc = c->F[p.level].gc;
  k.H = c->F[p.level].H;
  k.lc = p.lc;
  k.fd = p.fd;
  k.invM = p.invM;
  k.r = p.r;
  k.p_new = p.p_new;
  k.rf = p.rf;
  k.s_rz = p.s_rz;
  k.s_rz_prev = p.s_rz_prev;
  k.red = make_red(c, p.s_out0, p.s_out1, p.s_out2);
  const bool fin = p.level == c->maxlevel;
  switch (p.epi) {
    case EPI_PLAIN: return run_pf<EPI_PLAIN, false>(c, k, fin);
    case EPI_RESIDUAL: return run_pf<EPI_RESIDUAL, false>(c, k, fin);
    case EPI_PCG: return run_pf<EPI_PCG, false>(c, k, fin);
    case EPI_FAS: return run_pf<EPI_FAS, false>(c, k, fin);
  }
  return HPC_ERR_ARG;
}

int launch_pf_diag(hpc_ctx* c, int level, double lc, double* out) {
  PfK k{};
  k.g = c->L[level];
  k.sg = strip_geo(k.g);
  k.epi = EPI_PLAIN;
  k.src = c->F[level].d;
  k.out = out;
  k.gc = c->F[level].gc;
  k.H = c->F[level].H;
  k.lc = lc;
  k.red = make_red(c, -1, -1, -1);
  return run_pf<EPI_PLAIN, true>(c, k, false);
}

}  // namespace hpc
