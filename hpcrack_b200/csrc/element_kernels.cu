// Element-operator kernels: mechanical K(d) u and diag K(d), phase-field A_d x and diag A_d, with
// fused epilogues (residual, (p, K p), FAS right-hand side, reactions).
//
// Tiling ("warp strip"): a warp owns a strip of 32 node columns in x (31 elements, 30 output
// nodes), wy element rows in y (wy-1 output node rows) and cz output node planes in z, and
// streams it row by row, layer by layer.  The strip shape (wy, cz) is chosen per level: long strips
// on large levels (little recomputation at strip edges), short ones on small levels, where the
// serial chain of elements a warp computes would otherwise set the kernel's duration.  Node rows
// are staged into a per-warp shared-memory ring with cp.async two rows ahead of use, so
// global-memory latency never sits on the element math.
// Per row step a lane computes one element from the staged rows; x-neighbour contributions are
// combined with one shuffle, y-neighbours through registers (the previous row's upper-face sums)
// and z-neighbours through a per-warp shared-memory carry of the previous layer's upper faces.
// Every node is written once, by the warp whose output range owns it, with a fixed summation
// order: no atomics, no block-wide barriers, deterministic results.  Warps stride over the strip
// list (persistent grid).
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "device_common.cuh"
#include "internal.h"

namespace hpc {

constexpr int kWarps = 4;    // warps per block
// Largest strip height in element rows (wy - 1 output node rows).  16-row strips (half the y
// recomputation) ran the 257^3 FP64 apply at 1.33 ms against 1.07 ms with 8 rows: measured and dropped.
constexpr int kWY = 8;
constexpr int kOX = 30;      // output nodes per strip in x (lanes 1..30)
constexpr int kRowW = 33;    // staged row width (32 lanes + the x+1 read of lane 31)
constexpr int kRing = 4;     // staged node rows in flight / in use per warp

struct StripGeo {
  int tx, ty, tz;            // strips per axis
  int wy, cz;                // element rows (2..kWY) and output planes per strip
  long long nstrips;
};

inline StripGeo strip_geo(const LevelGeo& g, int wy, int cz, int ox = kOX) {
  StripGeo s;
  s.wy = wy;
  s.cz = cz;
  s.tx = (g.nx + ox - 1) / ox;
  s.ty = (g.ny + wy - 2) / (wy - 1);
  s.tz = (g.nz + cz - 1) / cz;
  s.nstrips = (long long)s.tx * s.ty * s.tz;
  return s;
}

// Strip shape of a level by a latency model of the element math: the FP64 unit of an SM
// sub-partition finishes one element per fixed time whether one or several warps feed it, so a
// level's duration is set by the longest chain of elements one sub-partition computes,
//   wy * (cz + 1) elements per strip  x  ceil(strips / sub-partitions).
// Short strips shorten the chain but recompute more strip-edge elements; the model picks the
// shape with the shortest chain (ties: the least recomputation).
inline StripGeo choose_strips(const LevelGeo& g, long long subpartitions, int ox = kOX) {
  static const int wys[] = {8, 4, 2};
  static const int czs[] = {32, 16, 8, 4, 2};
  StripGeo best{};
  long long best_chain = -1, best_work = 0;
  for (int wy : wys)
    for (int cz : czs) {
      const StripGeo s = strip_geo(g, wy, cz, ox);
      const long long per = (long long)wy * (cz + 1);
      const long long chain = per * ((s.nstrips + subpartitions - 1) / subpartitions);
      const long long work = per * s.nstrips;
      if (best_chain < 0 || chain < best_chain || (chain == best_chain && work < best_work)) {
        best = s;
        best_chain = chain;
        best_work = work;
      }
    }
  return best;
}

// ------------------------------------------------------------------------------------------
// cp.async staging (8-byte copies, zero fill outside the grid)
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 4 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_el(double* smem, const double* gmem, bool pred) { cp_async8(smem, gmem, pred); }
__device__ __forceinline__ void cp_async_el(float* smem, const float* gmem, bool pred) { cp_async4(smem, gmem, pred); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait2() { asm volatile("cp.async.wait_group 2;\n" ::: "memory"); }

// A strip's staged stream: for each layer kk = z0-1 .. zend, node rows y = y0-1 .. y0-1+wy
// (rows = wy+1 rows), each row holding NF fields on the two planes kk and kk+1.  Stream row s sits in
// ring slot s % kRing at ring[((slot*NF + f)*2 + c)*kRowW + lane].
template <int NF, typename T = double>
struct Stream {
  T* ring;
  const T* const* fields;  // NF global arrays (node-indexed)
  int x, y0, z0, nlayers, total, rows;
  const LevelGeo* g;

  __device__ __forceinline__ void issue(int s, int lane) {
    if (s < total) {
      const int li = s / rows, r = s - li * rows;
      const int kk = z0 - 1 + li, y = y0 - 1 + r;
      const int slot = s & (kRing - 1);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int z = kk + c;
        const bool ok = x >= 0 && x < g->nx && y >= 0 && y < g->ny && z >= 0 && z < g->nz;
        const long long n = ok ? (long long)x + (long long)y * g->px + (long long)z * g->plane : 0;
#pragma unroll
        for (int f = 0; f < NF; ++f) cp_async_el(ring + ((slot * NF + f) * 2 + c) * kRowW + lane, fields[f] + n, ok);
      }
    }
    cp_async_commit();
  }
  // Row s has landed for every lane of the warp (this lane's copies, then the warp barrier).
  __device__ __forceinline__ bool wait(int) const {
    cp_async_wait2();
    __syncwarp();
    return true;
  }
  __device__ __forceinline__ T at(int s, int f, int c, int col) const {
    return ring[(((s & (kRing - 1)) * NF + f) * 2 + c) * kRowW + col];
  }
};

// ------------------------------------------------------------------------------------------
// TMA staging (cp.async.bulk.tensor): one elected lane per warp copies a whole staged row - the 3
// vector components on the two planes kk, kk+1, x from xs to xs + BX - 1 - with one tensor copy into
// the warp's ring slot, completion counted on the slot's mbarrier; every lane waits on the barrier's
// phase.  The copy's x start must be a multiple of 16 bytes, so it starts at xs = the strip's first
// column (x0 - 1) rounded down to 16 bytes, the box is BX wide (33 columns plus that offset, rounded
// up to 16 bytes) and the lanes index from the offset.  Out-of-range coordinates (x < 0, x >= px,
// y = -1 or ny, z = -1 or nz) read zeros, as the cp.async staging's zero fill does; columns nx .. px-1
// are padding slots, zero in every vector.  Loads only, no multicast, this GPU's own memory.
// ------------------------------------------------------------------------------------------
template <typename T> struct TmaShape;
template <> struct TmaShape<float> { static constexpr int BX = 36; };   // 144 B; offset <= 3
template <> struct TmaShape<double> { static constexpr int BX = 34; };  // 272 B; offset <= 1
template <typename T>
constexpr int tma_slot_bytes() { return ((3 * 2 * TmaShape<T>::BX * (int)sizeof(T)) + 127) / 128 * 128; }
constexpr int kTmaHead = 128;              // per warp: 4 mbarriers, padded to the slots' 128-B alignment
constexpr unsigned kTmaWaitPolls = 1u << 24;  // far above any copy's latency; then the kernel reports
template <typename T>
__host__ __device__ constexpr size_t tma_warp_bytes(int wy) {
  return (size_t)kTmaHead + (size_t)kRing * tma_slot_bytes<T>() + (size_t)(wy - 1) * 3 * 32 * sizeof(T);
}

// The copy's inner extent is a multiple of 16 bytes and covers 33 columns after any offset below 16
// bytes; ring slots and every warp's share of shared memory stay on 128-byte boundaries.
static_assert(TmaShape<float>::BX * 4 % 16 == 0 && TmaShape<float>::BX >= 33 + 3, "float box");
static_assert(TmaShape<double>::BX * 8 % 16 == 0 && TmaShape<double>::BX >= 33 + 1, "double box");
static_assert(tma_warp_bytes<float>(2) % 128 == 0 && tma_warp_bytes<float>(4) % 128 == 0 &&
                  tma_warp_bytes<float>(8) % 128 == 0, "float warp share");
static_assert(tma_warp_bytes<double>(2) % 128 == 0 && tma_warp_bytes<double>(4) % 128 == 0 &&
                  tma_warp_bytes<double>(8) % 128 == 0, "double warp share");
static_assert(kWY == 8, "the warp-share alignment above is checked for strip heights 2, 4 and 8");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

template <typename T>
struct TmaStream {
  static constexpr int BX = TmaShape<T>::BX;
  static constexpr int SLOT = tma_slot_bytes<T>() / (int)sizeof(T);  // elements per ring slot
  T* ring;
  uint64_t* bars;
  const CUtensorMap* map;
  int xs, off, y0, z0, nlayers, total, rows;
  unsigned base;  // rows this warp staged before the strip: the slot and phase of row s are base + s's
  double* err;

  __device__ __forceinline__ void issue(int s, int lane) const {
    if (lane != 0 || s >= total) return;
    const int li = s / rows, r = s - li * rows;
    const int kk = z0 - 1 + li, y = y0 - 1 + r;
    const unsigned g = base + (unsigned)s;
    const uint32_t bar = smem_u32(bars + (g & (kRing - 1)));
    const uint32_t dst = smem_u32(ring + (size_t)(g & (kRing - 1)) * SLOT);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(3 * 2 * BX * (int)sizeof(T))
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(dst),
        "l"(map), "r"(xs), "r"(y), "r"(kk), "r"(0), "r"(bar)
        : "memory");
  }
  // Waits for row s; a wait that runs out sets *err and returns false (the kernel then stops).
  __device__ __forceinline__ bool wait(int s) const {
    const unsigned g = base + (unsigned)s;
    const uint32_t bar = smem_u32(bars + (g & (kRing - 1)));
    const uint32_t parity = (g / kRing) & 1u;
    for (unsigned i = 0; i < kTmaWaitPolls; ++i) {
      uint32_t ok;
      asm volatile(
          "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}\n"
          : "=r"(ok)
          : "r"(bar), "r"(parity)
          : "memory");
      if (ok) return true;
    }
    if (err) *err = 1.0;
    return false;
  }
  __device__ __forceinline__ T at(int s, int f, int c, int col) const {
    return ring[(size_t)((base + (unsigned)s) & (kRing - 1)) * SLOT + (f * 2 + c) * BX + off + col];
  }
};

// ------------------------------------------------------------------------------------------
// mechanical
// ------------------------------------------------------------------------------------------
template <typename T>
struct MechKT {
  LevelGeo g;
  LevelGeo gf;  // fine level (FAS)
  StripGeo sg;
  const T* fields[6];  // staged: u0,u1,u2 then K,G,d (finest) or Ke,Ge (coarse)
  T* out;
  const int8_t* choice;
  double small_k;
  T* fu;
  int set_fnorm;
  const T* invM;
  const T* rf;
  const T* gpm;  // finest level, precomputed Gauss-point moduli: K - 2G/3 at [g * n + e], G at [(8 + g) * n + e]
  RedTarget red;
  double* err;   // tensor-core kernel / TMA staging: set to 1 when a bounded wait ran out
  alignas(64) CUtensorMap tmap;  // TMA staging: the staged vector as {px, ny, nz, 3} (finest applies)
};
using MechK = MechKT<double>;

// d clamped to [0, 1] (K_G_d_g, material_gauss_point.cpp:51-54), decided on the bit pattern:
// negative values (sign bit set) give 0, values above 1 give 1.
__device__ __forceinline__ double clamp01(double v) {
  const long long b = __double_as_longlong(v);
  return b < 0 ? 0.0 : (b > 0x3FF0000000000000LL ? 1.0 : v);
}
__device__ __forceinline__ float clamp01(float v) {
  const int b = __float_as_int(v);
  return b < 0 ? 0.0f : (b > 0x3F800000 ? 1.0f : v);
}

// Per-Gauss-point moduli times wg (MP_all_GAUSS_Point, mechanical_pcg.cpp:26-61), finest level:
// trilinear nodal K, G, d with the zero rule, clamp and degradation by regime.
template <typename T>
__device__ __forceinline__ void mech_moduli_finest(const T (&Kn)[8], const T (&Gn)[8], const T (&dn)[8], int ch,
                                                   T small_k, T wg, const SFt<T>& s, T (&Kw)[8], T (&Gw)[8]) {
  T Kg[8], Gg[8];
  gp_material(Kn, s, Kg);
  gp_material(Gn, s, Gg);
  if (ch == 2) {
#pragma unroll
    for (int g = 0; g < 8; ++g) {
      Kw[g] = Kg[g] * wg;
      Gw[g] = Gg[g] * wg;
    }
  } else {
    T dg[8];
    gp_material(dn, s, dg);
    const T one_k = T(1) - small_k;
#pragma unroll
    for (int g = 0; g < 8; ++g) {
      const T om = T(1) - clamp01(dg[g]);
      const T gd = fma(one_k * om, om, small_k);
      Kw[g] = (ch == 0 ? gd * Kg[g] : Kg[g]) * wg;
      Gw[g] = (gd * Gg[g]) * wg;
    }
  }
}

// Assembly of one row step's element forces f (lane: element x0-1+lane of row ey, layer kk) into
// nodes: x-neighbours by one shuffle, y-neighbours through the register carry yp, z-neighbours
// through the warp's shared-memory carry zc; then the epilogue of output node (x, ey, kk) when this
// row step completes it.
template <typename T, int EPI, class ST>
__device__ __forceinline__ void assemble_row(const MechKT<T>& k, const ST& st, int si, int lane, int x,
                                             int ey, int kk, int z0, int rr, const T (&f)[3][8], T (&yp)[2][3],
                                             T* zc, double& red0, double& red1, double& red2) {
  // ---- combine x-neighbours: node x gets own a=0 corners + left lane's a=1 corners
  T X[2][2][3];  // [b][c][m]
#pragma unroll
  for (int c = 0; c < 2; ++c)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        const T left = __shfl_up_sync(kFull, f[m][1 + 2 * b + 4 * c], 1);
        X[b][c][m] = f[m][2 * b + 4 * c] + (lane > 0 ? left : T(0));
      }
  if (rr >= 1) {
    const int orow = rr - 1;
    T tot[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      T* zp = zc + (orow * 3 + m) * 32 + lane;
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
        // a slab's ghost planes keep the sums as they are (a select: ghost values may be anything)
        const bool own = owned_plane(k.g, kk);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          T fv = k.fu[n + m * N];
          if (k.set_fnorm && fix[m]) {
            fv = tot[m];
            k.fu[n + m * N] = fv;
          }
          if (k.red.slot[0] >= 0) {  // sums nobody reads are skipped
            const double s0 = fma((double)fv, (double)fv, red0);
            red0 = own ? s0 : red0;
          }
          const T rv = fix[m] ? T(0) : fv - tot[m];
          k.out[n + m * N] = rv;
          if (k.invM) {
            const double s1 = fma((double)rv, (double)(rv * k.invM[n + m * N]), red1);
            red1 = own ? s1 : red1;
          }
          if (k.red.slot[2] >= 0) {
            const double s2 = fma((double)rv, (double)rv, red2);
            red2 = own ? s2 : red2;
          }
        }
      } else if (EPI == EPI_PCG) {  // w = K p, (p, w)
        const bool own = owned_plane(k.g, kk);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          k.out[n + m * N] = tot[m];
          const double s0 = fma((double)st.at(si - 1, m, 0, lane), (double)tot[m], red0);
          red0 = own ? s0 : red0;
        }
      } else if (EPI == EPI_FAS) {
        // coarsen_f_standard_routine (multigrid_intergrid.cpp:124-342) fused with the coarse apply;
        // a slab's lower ghost plane has no fine plane below it (its value comes from the neighbour)
        const int fz = 2 * kk + k.g.zsh;
#pragma unroll
        for (int m = 0; m < 3; ++m)
          k.out[n + m * N] =
              tot[m] + (fz >= 0 ? full_weight(k.gf, k.rf + (long long)m * k.gf.n, 2 * x, 2 * ey, fz) : T(0));
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

// T = double: the plain form; T = float: the precision form's V-cycle (reductions stay FP64).
// GPM: the finest level's Gauss-point moduli come precomputed (gp_material_kernel) instead of being
// interpolated from the staged nodal K, G, d in every apply.
// TMA: the finest applies on precomputed moduli stage their rows with tensor copies (TmaStream)
// instead of per-lane cp.async; the same values reach the same arithmetic, so the same bits.
template <typename T, bool FINEST, int EPI, bool DIAG, bool ISO, bool GPM = false, bool TMA = false>
__global__ void __launch_bounds__(kWarps * 32) mech_kernel(const __grid_constant__ MechKT<T> k) {
  constexpr int NU = DIAG ? 0 : 3;
  constexpr int NF = NU + (FINEST ? (GPM ? 0 : 3) : 2);
  static_assert(!TMA || (FINEST && GPM && !DIAG), "TMA staging serves the finest applies on precomputed moduli");
  extern __shared__ __align__(128) unsigned char mech_smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  // per warp: [TMA: 4 mbarriers] the staging ring, then the z-carry of the strip's wy - 1 output rows
  const size_t wbytes = TMA ? tma_warp_bytes<T>(k.sg.wy)
                            : (size_t)(kRing * NF * 2 * kRowW + (k.sg.wy - 1) * 3 * 32) * sizeof(T);
  // TMA: ring slots on 128-byte boundaries (the launch adds 128 bytes for this alignment)
  unsigned char* base = TMA ? mech_smem + ((128u - (smem_u32(mech_smem) & 127u)) & 127u) : mech_smem;
  unsigned char* wbase = base + (size_t)wib * wbytes;
  T* ring = reinterpret_cast<T*>(wbase + (TMA ? kTmaHead : 0));
  T* zc = ring + (TMA ? (size_t)kRing * TmaStream<T>::SLOT : (size_t)kRing * NF * 2 * kRowW);  // [row][comp][lane]
  uint64_t* bars = reinterpret_cast<uint64_t*>(wbase);
  if constexpr (TMA) {
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < kRing; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bars + i)) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
  }
  const SFt<T> s = make_sf<T>(k.g);
  double red0 = 0.0, red1 = 0.0, red2 = 0.0;
  const long long nwarps_total = (long long)gridDim.x * kWarps;
  const T* fptr[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) fptr[f] = k.fields[f];
  unsigned staged = 0;  // rows this warp staged so far (TMA: slot and barrier phase bookkeeping)

  for (long long strip = (long long)blockIdx.x * kWarps + wib; strip < k.sg.nstrips; strip += nwarps_total) {
    const int sx = (int)(strip % k.sg.tx);
    const long long rest = strip / k.sg.tx;
    const int sy = (int)(rest % k.sg.ty);
    const int sz = (int)(rest / k.sg.ty);
    const int wy = k.sg.wy, rows = wy + 1;
    const int x0 = sx * kOX, y0 = sy * (wy - 1), z0 = sz * k.sg.cz;
    const int x = x0 - 1 + lane;
    const int zend = min(z0 + k.sg.cz - 1, k.g.nz - 1);
    const int nlayers = zend - z0 + 2;
    // one strip, whichever staging: rows issued two ahead, each row waited for before use
    auto run_strip = [&](auto& st) -> bool {
      st.issue(0, lane);
      st.issue(1, lane);
      T yp[2][3];
      for (int si = 0; si < st.total; ++si) {
        st.issue(si + 2, lane);
        if (!st.wait(si)) return false;
        const int li = si / rows, r = si - li * rows;
        const int kk = z0 - 1 + li;
        if (r == 0) {
#pragma unroll
          for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int m = 0; m < 3; ++m) yp[c][m] = T(0);
          __syncwarp();
          continue;
        }
        const int rr = r - 1, ey = y0 - 1 + rr;
        if (EPI == EPI_RESIDUAL && rr >= 1 && kk >= z0 && lane >= 1 && lane <= 30 && x < k.g.nx && ey < k.g.ny) {
          // the epilogue reads f and M^-1 of this row's output node: start them towards L2 now, so
          // their latency overlaps the element math instead of following it
          const long long n = (long long)x + (long long)ey * k.g.px + (long long)kk * k.g.plane;
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            asm volatile("prefetch.global.L2 [%0];" ::"l"(k.fu + n + m * k.g.n));
            if (k.invM) asm volatile("prefetch.global.L2 [%0];" ::"l"(k.invM + n + m * k.g.n));
          }
        }
        // ---- element (x, ey, kk) from stream rows si-1 (y = ey) and si (y = ey+1)
        T f[3][8];
        const bool valid = lane < 31 && x >= 0 && x <= k.g.nx - 2 && ey >= 0 && ey <= k.g.ny - 2 && kk >= 0 &&
                           kk <= k.g.nz - 2;
        if (valid) {
          T Kw[8], Gw[8];
          // ISO: the 1/h^2 of the two gradients goes into the Gauss weight (see sf_forward)
          const T wg = ISO ? T(k.g.wg) * (s.ih[0] * s.ih[0]) : T(k.g.wg);
          if (FINEST && GPM) {
            const long long e = (long long)x + (long long)ey * k.g.px + (long long)kk * k.g.plane;
#pragma unroll
            for (int g = 0; g < 8; ++g) {
              Kw[g] = k.gpm[(long long)g * k.g.n + e];
              Gw[g] = k.gpm[(long long)(8 + g) * k.g.n + e];
            }
          } else if (FINEST) {
            T Kn[8], Gn[8], dn[8];
#pragma unroll
            for (int n = 0; n < 8; ++n) {
              const int a = n & 1, b = (n >> 1) & 1, c = n >> 2;
              const int srow = b ? si : si - 1;
              Kn[n] = st.at(srow, NU + 0, c, lane + a);
              Gn[n] = st.at(srow, NU + 1, c, lane + a);
              dn[n] = st.at(srow, NU + 2, c, lane + a);
            }
            const long long e = (long long)x + (long long)ey * k.g.px + (long long)kk * k.g.plane;
            mech_moduli_finest(Kn, Gn, dn, k.choice[e], T(k.small_k), wg, s, Kw, Gw);
          } else {
            const T K = st.at(si - 1, NU + 0, 0, lane) * wg, G = st.at(si - 1, NU + 1, 0, lane) * wg;
#pragma unroll
            for (int g = 0; g < 8; ++g) {
              Kw[g] = K;
              Gw[g] = G;
            }
          }
          if constexpr (DIAG) {
            mech_element_diag(Kw, Gw, s, f);
          } else {
            T u[3][8];
#pragma unroll
            for (int n = 0; n < 8; ++n) {
              const int a = n & 1, b = (n >> 1) & 1, c = n >> 2;
              const int srow = b ? si : si - 1;
#pragma unroll
              for (int m = 0; m < 3; ++m) u[m][n] = st.at(srow, m, c, lane + a);
            }
            mech_element<ISO, T, FINEST && GPM>(u, Kw, Gw, s, f);
          }
        } else {
#pragma unroll
          for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int n = 0; n < 8; ++n) f[m][n] = T(0);
        }
        assemble_row<T, EPI>(k, st, si, lane, x, ey, kk, z0, rr, f, yp, zc, red0, red1, red2);
        __syncwarp();
      }
      return true;
    };
    if constexpr (TMA) {
      constexpr int A = 16 / (int)sizeof(T);  // columns per 16 bytes: the copy's x start is a multiple
      const int xs = x0 - 1 >= 0 ? (x0 - 1) / A * A : -A;
      TmaStream<T> st{ring, bars, &k.tmap, xs, (x0 - 1) - xs, y0, z0, nlayers, nlayers * rows, rows, staged, k.err};
      if (!run_strip(st)) break;
      staged += (unsigned)st.total;
    } else {
      Stream<NF, T> st{ring, fptr, x, y0, z0, nlayers, nlayers * rows, rows, &k.g};
      run_strip(st);
    }
  }
  if (EPI == EPI_RESIDUAL || EPI == EPI_PCG) {
    double v[3] = {red0, red1, red2};
    grid_reduce<3>(v, k.red);
  }
}


// ------------------------------------------------------------------------------------------
// Tensor-core element contraction (precision form, FP32 with TF32 operands)
// ------------------------------------------------------------------------------------------
// The same strips and node assembly as mech_kernel, with the element algebra as two small GEMMs on
// the 5th-generation tensor cores.  A block's 4 warps march 4 strips in lockstep, so one row step
// gives 128 elements = 128 rows of an MMA tile (TMEM lane 32w+l = element of lane l of warp w):
//   strains  D1[e][(g,s)] = sum_k U[e][k] B[(g,s)][k]     128 x 48, K = 24 (3 MMAs of K = 8)
//   stresses S[e][(g,s)]  = Hooke's law per Gauss point g with that point's moduli (CUDA cores)
//   forces   D2[e][k]     = sum_(g,s) S[e][(g,s)] B[(g,s)][k]   128 x 24 (N padded to 32), K = 48
// k = m*8 + n indexes the element's 24 DoFs (component m, node n = a + 2b + 4c), s the 6 engineering
// strains (xx, yy, zz, xy, xz, yz); B holds the reference-coordinate shape-function derivatives at
// the 2x2x2 Gauss points (isotropic spacing: the material carries 1/h^2 and the Gauss weight, as in
// the stencil kernels).  Operands are staged in shared memory in the canonical K-major layout
// without swizzle (a core matrix = 8 rows x 16 bytes, contiguous); one thread issues the MMAs and
// commits them to an mbarrier; every thread reads its own element's row back from TMEM.
// TF32 keeps 10 mantissa bits of each operand: an approximation of the FP32 operator at the 1e-3
// level, used only inside the preconditioning V-cycle of the flexible-PCG precision form.
constexpr int kTcCols = 128;                 // TMEM columns per block: D1 at 0..47, D2 at 64..95
constexpr int kTcD2 = 64;
constexpr int kTcABytes = 12 * 128 * 16;     // A tile: 128 rows, K up to 48 (12 chunks of 4 values)
constexpr int kTcB1Bytes = 6 * 48 * 16;      // B for the strains: 48 rows, K = 24
constexpr int kTcB2Bytes = 12 * 32 * 16;     // B for the forces: 32 rows (24 used), K = 48
constexpr int kTcHead = kTcABytes + kTcB1Bytes + kTcB2Bytes + 16;  // + mbarrier and TMEM address
constexpr unsigned kTcWaitPolls = 1u << 24;  // ~0.5 s of polling: far above any MMA's latency

// Shape-function derivative d N_n / d xi_j at Gauss point g, reference coordinates of the element.
__device__ __forceinline__ float tc_dn(int n, int j, int g, float t0, float t1) {
  const int a[3] = {n & 1, (n >> 1) & 1, n >> 2};
  const float tg[3] = {(g & 1) ? t1 : t0, ((g >> 1) & 1) ? t1 : t0, (g >> 2) ? t1 : t0};
  float v = 1.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float shape = a[d] ? tg[d] : 1.f - tg[d];
    v *= d == j ? (a[d] ? 1.f : -1.f) : shape;
  }
  return v;
}
// Strain-displacement entry: row (g, s) = g*6 + s, column k = m*8 + n.
__device__ __forceinline__ float tc_b(int row, int k, float t0, float t1) {
  const int g = row / 6, sd = row % 6, m = k >> 3, n = k & 7;
  // derivative direction of component m in strain sd (-1: the component does not enter it):
  // xx: u_x,x  yy: u_y,y  zz: u_z,z  xy: u_x,y + u_y,x  xz: u_x,z + u_z,x  yz: u_y,z + u_z,y
  int j = -1;
  if (sd < 3) j = m == sd ? sd : -1;
  else if (sd == 3) j = m == 0 ? 1 : (m == 1 ? 0 : -1);
  else if (sd == 4) j = m == 0 ? 2 : (m == 2 ? 0 : -1);
  else j = m == 1 ? 2 : (m == 2 ? 1 : -1);
  return j < 0 ? 0.f : tc_dn(n, j, g, t0, t1);
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);  // version 1, no swizzle
}
// kind::tf32, F32 accumulate, both operands K-major, M = 128.
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
  for (unsigned i = 0; i < kTcWaitPolls; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16], int o) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
  (void)o;
}
__device__ __forceinline__ void tc_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Row steps a strip of the strip list takes (layers of its z-slab x (wy + 1) staged rows); 0 past the list.
__device__ __forceinline__ int strip_steps(const StripGeo& sg, const LevelGeo& g, long long strip) {
  if (strip >= sg.nstrips) return 0;
  const int sz = (int)(strip / ((long long)sg.tx * sg.ty));
  const int z0 = sz * sg.cz;
  const int zend = min(z0 + sg.cz - 1, g.nz - 1);
  return (zend - z0 + 2) * (sg.wy + 1);
}

template <bool FINEST, int EPI>
__global__ void __launch_bounds__(kWarps * 32) mech_tc_kernel(MechKT<float> k) {
  using T = float;
  constexpr int NU = 3;
  constexpr int NF = NU + (FINEST ? 0 : 2);  // the finest level reads precomputed Gauss-point moduli
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  float* As = reinterpret_cast<float*>(tc_smem);
  float* B1s = reinterpret_cast<float*>(tc_smem + kTcABytes);
  float* B2s = reinterpret_cast<float*>(tc_smem + kTcABytes + kTcB1Bytes);
  uint64_t* bar = reinterpret_cast<uint64_t*>(tc_smem + kTcABytes + kTcB1Bytes + kTcB2Bytes);
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  T* ring = reinterpret_cast<T*>(tc_smem + kTcHead) + (size_t)wib * (kRing * NF * 2 * kRowW + (k.sg.wy - 1) * 3 * 32);
  T* zc = ring + kRing * NF * 2 * kRowW;
  const SFt<T> s = make_sf<T>(k.g);
  const uint32_t sA = (uint32_t)__cvta_generic_to_shared(As), sB1 = (uint32_t)__cvta_generic_to_shared(B1s);
  const uint32_t sB2 = (uint32_t)__cvta_generic_to_shared(B2s), sbar = (uint32_t)__cvta_generic_to_shared(bar);

  // ---- set-up: the two B operands, the mbarrier, 128 TMEM columns
  for (int i = tid; i < 48 * 24; i += blockDim.x) {
    const int r = i / 24, kk = i - r * 24;
    B1s[(kk >> 2) * 48 * 4 + r * 4 + (kk & 3)] = tc_b(r, kk, s.t[0], s.t[1]);
  }
  for (int i = tid; i < 32 * 48; i += blockDim.x) {
    const int r = i / 48, kk = i - r * 48;
    B2s[(kk >> 2) * 32 * 4 + r * 4 + (kk & 3)] = r < 24 ? tc_b(kk, r, s.t[0], s.t[1]) : 0.f;
  }
  if (wib == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(taddr_s)),
                 "r"(kTcCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sbar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *taddr_s;
  const uint32_t trow = tmem + ((uint32_t)(wib * 32) << 16);  // this warp's 32 TMEM lanes

  const T wg = T(k.g.wg) * (s.ih[0] * s.ih[0]);  // isotropic spacing: 1/h^2 in the Gauss weight
  double red0 = 0.0, red1 = 0.0, red2 = 0.0;
  const T* fptr[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) fptr[f] = k.fields[f];
  uint32_t phase = 0;
  int bad = 0, aborted = 0;
  const long long nblk_strips = (k.sg.nstrips + kWarps - 1) / kWarps;

  for (long long cs = blockIdx.x; cs < nblk_strips && !aborted; cs += gridDim.x) {
    const long long strip = cs * kWarps + wib;
    int steps = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) steps = max(steps, strip_steps(k.sg, k.g, cs * kWarps + w));
    const bool active = strip < k.sg.nstrips;
    const long long sref = active ? strip : cs * kWarps;  // inactive warps follow the block's first strip
    const int sx = (int)(sref % k.sg.tx);
    const long long rest = sref / k.sg.tx;
    const int sy = (int)(rest % k.sg.ty);
    const int sz = (int)(rest / k.sg.ty);
    const int wy = k.sg.wy, rows = wy + 1;
    const int x0 = sx * kOX, y0 = sy * (wy - 1), z0 = sz * k.sg.cz;
    const int x = x0 - 1 + lane;
    const int zend = min(z0 + k.sg.cz - 1, k.g.nz - 1);
    Stream<NF, T> st{ring, fptr, x, y0, z0, zend - z0 + 2, 0, rows, &k.g};
    st.total = active ? st.nlayers * rows : 0;
    st.issue(0, lane);
    st.issue(1, lane);
    T yp[2][3];
    for (int si = 0; si < steps; ++si) {
      st.issue(si + 2, lane);
      cp_async_wait2();
      __syncwarp();
      const int li = si / rows, r = si - li * rows;  // the same for the 4 strips: equal shapes
      const int kk = z0 - 1 + li;
      if (r == 0) {
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
          for (int m = 0; m < 3; ++m) yp[c][m] = T(0);
        __syncwarp();
        continue;
      }
      const bool mine = si < st.total;  // this warp's strip still has this row step
      const int rr = r - 1, ey = y0 - 1 + rr;
      const bool valid = mine && lane < 31 && x >= 0 && x <= k.g.nx - 2 && ey >= 0 && ey <= k.g.ny - 2 &&
                         kk >= 0 && kk <= k.g.nz - 2;
      const int row = wib * 32 + lane;
      // this element's moduli, loaded now so that their latency overlaps the strain MMAs
      T Kw[8], Gw[8];
      if (valid) {
        if (FINEST) {
          const long long el = (long long)x + (long long)ey * k.g.px + (long long)kk * k.g.plane;
#pragma unroll
          for (int g = 0; g < 8; ++g) {
            Kw[g] = k.gpm[(long long)g * k.g.n + el];
            Gw[g] = k.gpm[(long long)(8 + g) * k.g.n + el];
          }
        } else {
          const T K = st.at(si - 1, NU + 0, 0, lane) * wg, G = st.at(si - 1, NU + 1, 0, lane) * wg;
#pragma unroll
          for (int g = 0; g < 8; ++g) {
            Kw[g] = K;
            Gw[g] = G;
          }
        }
      } else {
#pragma unroll
        for (int g = 0; g < 8; ++g) Kw[g] = Gw[g] = T(0);
      }
      // ---- A = the element's 24 displacement values (zeros for lanes without an element)
      {
        T u[24];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
          const int a = n & 1, b = (n >> 1) & 1, c = n >> 2;
          const int srow = b ? si : si - 1;
#pragma unroll
          for (int m = 0; m < 3; ++m) u[m * 8 + n] = valid ? st.at(srow, m, c, lane + a) : T(0);
        }
#pragma unroll
        for (int kc = 0; kc < 6; ++kc)
          *reinterpret_cast<float4*>(As + kc * 512 + row * 4) =
              make_float4(u[4 * kc], u[4 * kc + 1], u[4 * kc + 2], u[4 * kc + 3]);
      }
      fence_async_smem();
      tc_fence_before();
      if (__syncthreads_or(bad)) { aborted = 1; break; }
      if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < 3; ++q)
          tc_mma(tmem, tc_desc(sA + q * 4096, 2048, 128), tc_desc(sB1 + q * 1536, 768, 128), tc_idesc(48), q > 0);
        tc_commit(sbar);
      }
      if (!tc_wait(sbar, phase)) bad = 1;
      phase ^= 1u;
      tc_fence_after();
      // ---- strains of the element at its 8 Gauss points -> stresses
      float e[48];
      {
        float t16[16];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          tc_ld16(trow + q * 16, t16, q);
          tc_wait_ld();
#pragma unroll
          for (int i = 0; i < 16; ++i) e[q * 16 + i] = t16[i];
        }
      }
      {
#pragma unroll
        for (int g = 0; g < 8; ++g) {
          float* v = e + 6 * g;
          const T K = Kw[g], G = Gw[g];
          const T tr = v[0] + v[1] + v[2];
          const T lt = (FINEST ? K : fmaf(T(-2.0 / 3.0), G, K)) * tr;  // the finest moduli hold K - 2G/3
          const T G2 = G + G;
          v[0] = fmaf(G2, v[0], lt);
          v[1] = fmaf(G2, v[1], lt);
          v[2] = fmaf(G2, v[2], lt);
          v[3] *= G;
          v[4] *= G;
          v[5] *= G;
        }
#pragma unroll
        for (int kc = 0; kc < 12; ++kc)
          *reinterpret_cast<float4*>(As + kc * 512 + row * 4) =
              make_float4(e[4 * kc], e[4 * kc + 1], e[4 * kc + 2], e[4 * kc + 3]);
      }
      fence_async_smem();
      tc_fence_before();
      if (__syncthreads_or(bad)) { aborted = 1; break; }
      if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int q = 0; q < 6; ++q)
          tc_mma(tmem + kTcD2, tc_desc(sA + q * 4096, 2048, 128), tc_desc(sB2 + q * 1024, 512, 128), tc_idesc(32),
                 q > 0);
        tc_commit(sbar);
      }
      if (!tc_wait(sbar, phase)) bad = 1;
      phase ^= 1u;
      tc_fence_after();
      T f[3][8];
      {
        float a16[16], a8[8];
        tc_ld16(trow + kTcD2, a16, 0);
        tc_ld8(trow + kTcD2 + 16, a8);
        tc_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) f[i >> 3][i & 7] = a16[i];
#pragma unroll
        for (int i = 0; i < 8; ++i) f[2][i] = a8[i];
      }
      tc_fence_before();
      if (mine) assemble_row<T, EPI>(k, st, si, lane, x, ey, kk, z0, rr, f, yp, zc, red0, red1, red2);
      __syncwarp();
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  if (aborted && tid == 0 && k.err) *k.err = 1.0;
  if (EPI == EPI_RESIDUAL || EPI == EPI_PCG) {
    double v[3] = {red0, red1, red2};
    grid_reduce<3>(v, k.red);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (wib == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols));
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

RedTarget make_red(hpc_ctx* c, int s0, int s1, int s2, int op) {
  RedTarget t;
  t.partials = c->partials;
  t.counter = c->counter;
  t.scal = c->scal;
  t.slot[0] = s0;
  t.slot[1] = s1;
  t.slot[2] = s2;
  if (c->slab) {
    c->red_slot[0] = s0;
    c->red_slot[1] = s1;
    c->red_slot[2] = s2;
    c->red_op = op;
    c->red_pending = 1;
  }
  return t;
}

// Per-kernel launch configuration (dynamic shared-memory opt-in and resident blocks per SM), set up
// on a kernel's first launch so that later launches - also those inside a stream capture - only
// enqueue work.
// Dynamic shared memory of a strip kernel as a function of the strip height wy: `fixed` bytes, then
// per warp a staging ring of `ring` elements and a z-carry of `row` elements per output row
// (wy - 1 rows), elements of `elem` bytes.
struct SmemPlan {
  size_t fixed, ring, row, elem;
  size_t bytes(int wy) const { return fixed + (size_t)kWarps * (ring + (size_t)(wy - 1) * row) * elem; }
};

// Per kernel and dynamic shared-memory size: the opt-in and resident blocks per SM, set up on first
// use so that later launches - also those inside a stream capture - only enqueue work.
struct KernelCfg {
  const void* fn;
  int device;
  size_t smem;
  int per_sm;
};
static std::mutex g_cfg_mu;
static KernelCfg g_cfg[512];
static int g_ncfg = 0;

template <class Kern>
static int kernel_cfg(Kern kern, size_t max_smem, size_t smem, int* per_sm_out) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_cfg_mu);
  for (int i = 0; i < g_ncfg; ++i)
    if (g_cfg[i].fn == (const void*)kern && g_cfg[i].device == dev && g_cfg[i].smem == smem) {
      *per_sm_out = g_cfg[i].per_sm;
      return HPC_OK;
    }
  // opt in always: the 48 KB default bounds static plus dynamic shared memory together, and the
  // kernels' own static share would push a dynamic size just below 48 KB over it
  {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(smem)");
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kWarps * 32, smem);
  if (e != cudaSuccess || per_sm <= 0) per_sm = 1;
  if (g_ncfg < 512) g_cfg[g_ncfg++] = KernelCfg{(const void*)kern, dev, smem, per_sm};
  *per_sm_out = per_sm;
  return HPC_OK;
}

// Strip shapes chosen by measurement (hpc_set_autotune), per kernel, device and level size; shared
// by every context of the process once measured.
struct TunedShape {
  const void* fn;
  int device, nx, ny, nz, wy, cz;
};
static std::mutex g_tune_mu;
static TunedShape g_tuned[512];
static int g_ntuned = 0;

static bool tuned_shape(const void* fn, int dev, const LevelGeo& g, StripGeo* out, int ox) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  for (int i = 0; i < g_ntuned; ++i) {
    const TunedShape& t = g_tuned[i];
    if (t.fn == fn && t.device == dev && t.nx == g.nx && t.ny == g.ny && t.nz == g.nz) {
      *out = strip_geo(g, t.wy, t.cz, ox);
      return true;
    }
  }
  return false;
}

static int grid_for(const StripGeo& sg, long long cap) {
  const long long need = (sg.nstrips + kWarps - 1) / kWarps;
  return (int)(need < cap ? need : cap);
}

// Times every candidate shape on the live arguments (element kernels are pure functions of their
// inputs: a repeated launch rewrites the same outputs and reductions) and keeps the fastest.
template <class Kern, class Args>
static int autotune_shape(hpc_ctx* c, Kern kern, Args a, const SmemPlan& plan, StripGeo* best, int ox) {
  static const int wys[] = {8, 4, 2};
  static const int czs[] = {32, 16, 8, 4, 2};
  cudaEvent_t e0, e1;
  HPC_CUDA(cudaEventCreate(&e0));
  HPC_CUDA(cudaEventCreate(&e1));
  float best_ms = 1e30f;
  *best = choose_strips(a.g, (long long)num_sms() * 4, ox);
  int rc = HPC_OK;
  for (int wy : wys) {
    for (int cz : czs) {
      a.sg = strip_geo(a.g, wy, cz, ox);
      const size_t smem = plan.bytes(wy);
      int per_sm = 1;
      if ((rc = kernel_cfg(kern, plan.bytes(kWY), smem, &per_sm))) break;
      const int grid = grid_for(a.sg, (long long)num_sms() * per_sm);
      if (grid <= 0 || (size_t)grid * 3 > c->partials_cap) continue;
      kern<<<grid, kWarps * 32, smem, c->stream>>>(a);
      cudaEventRecord(e0, c->stream);
      kern<<<grid, kWarps * 32, smem, c->stream>>>(a);
      kern<<<grid, kWarps * 32, smem, c->stream>>>(a);
      cudaEventRecord(e1, c->stream);
      c->launches += 3;
      cudaError_t e = cudaEventSynchronize(e1);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e != cudaSuccess) {
        rc = cuda_fail(e, "autotune launch");
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best_ms) {
        best_ms = ms;
        *best = a.sg;
      }
    }
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// Launches a strip kernel with the occupancy the device allows (persistent grid).  The strip shape
// of the level comes from the latency model (choose_strips), or - for a context with autotuning on -
// from a measurement (first use of a kernel on a level size, outside stream capture, kept for every
// autotuning context of the process).
// `units`: the strip-shape model's parallel units (0: the SM sub-partitions).
template <class Kern, class Args>
static int launch_strips(hpc_ctx* c, Kern kern, Args a, const SmemPlan& plan, int cls, int ox = kOX,
                         long long units = 0) {
  int rc = HPC_OK;
  if (units <= 0) units = (long long)num_sms() * 4;
  int dev = 0;
  cudaGetDevice(&dev);
  // Measured shapes serve only contexts with autotuning on: a context without it always takes the
  // model's shapes, so its results never depend on what another context measured.
  if (!c->autotune) {
    a.sg = choose_strips(a.g, units, ox);
  } else if (!tuned_shape((const void*)kern, dev, a.g, &a.sg, ox)) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) {
      if ((rc = autotune_shape(c, kern, a, plan, &a.sg, ox))) return rc;
      std::lock_guard<std::mutex> lock(g_tune_mu);
      if (g_ntuned < 512)
        g_tuned[g_ntuned++] = TunedShape{(const void*)kern, dev, a.g.nx, a.g.ny, a.g.nz, a.sg.wy, a.sg.cz};
    } else {
      a.sg = choose_strips(a.g, units, ox);
    }
  }
  const size_t smem = plan.bytes(a.sg.wy);
  int per_sm = 1;
  if ((rc = kernel_cfg(kern, plan.bytes(kWY), smem, &per_sm))) return rc;
  const int grid = grid_for(a.sg, (long long)num_sms() * per_sm);
  if (grid <= 0) return HPC_OK;
  if ((size_t)grid * 3 > c->partials_cap) return cuda_fail(cudaErrorInvalidValue, "partials buffer");
  timing_begin(c, cls);
  kern<<<grid, kWarps * 32, smem, c->stream>>>(a);
  timing_end(c, cls);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// Shapes measured so far (for reports): up to cap entries of {nx, ny, nz, wy, cz}.
int tuned_shapes(int* out5, int cap) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  int n = 0;
  for (int i = 0; i < g_ntuned && n < cap; ++i, ++n) {
    out5[5 * n + 0] = g_tuned[i].nx;
    out5[5 * n + 1] = g_tuned[i].ny;
    out5[5 * n + 2] = g_tuned[i].nz;
    out5[5 * n + 3] = g_tuned[i].wy;
    out5[5 * n + 4] = g_tuned[i].cz;
  }
  return n;
}

// Isotropic spacing (hx = hy = hz) selects the kernels that fold 1/h^2 into the material.
inline bool iso(const LevelGeo& g) { return g.hx == g.hy && g.hy == g.hz; }

// The staged vector of a finest apply as a TMA tensor {px, ny, nz, 3} (x fastest; the three components
// n apart), box {BX, 1, 2, 3}: one copy brings a row's three components on two planes.
using EncodeTiled = PFN_cuTensorMapEncodeTiled_v12000;
static EncodeTiled tensor_map_encoder() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q{};
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}
template <typename T>
static int encode_rows(const LevelGeo& g, const T* src, CUtensorMap* map) {
  EncodeTiled enc = tensor_map_encoder();
  if (!enc) {
    set_error("TMA staging: cuTensorMapEncodeTiled unavailable");
    return HPC_ERR_CUDA;
  }
  const cuuint64_t es = sizeof(T);
  const cuuint64_t dims[4] = {(cuuint64_t)g.px, (cuuint64_t)g.ny, (cuuint64_t)g.nz, 3};
  const cuuint64_t strides[3] = {(cuuint64_t)g.px * es, (cuuint64_t)g.plane * es, (cuuint64_t)g.n * es};
  const cuuint32_t box[4] = {(cuuint32_t)TmaShape<T>::BX, 1, 2, 3};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = enc(map, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                         const_cast<T*>(src), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("TMA staging: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return HPC_ERR_CUDA;
  }
  return HPC_OK;
}

template <bool F, int E, bool D, typename T = double>
static int run_mech(hpc_ctx* c, const MechKT<T>& k, bool tma = false) {
  const int cls = (F && E == EPI_PCG && !D) ? (sizeof(T) == 8 ? HPC_KC_MECH_PCG_FINEST : HPC_KC_MECH32_PCG_FINEST)
                                             : HPC_KC_NONE;
  if constexpr (F && !D) {
    if (k.gpm && tma) {  // precomputed Gauss-point moduli, rows staged by tensor copies
      const SmemPlan smem{128, (kTmaHead + (size_t)kRing * tma_slot_bytes<T>()) / sizeof(T), 3 * 32, sizeof(T)};
      if (iso(k.g)) return launch_strips(c, mech_kernel<T, F, E, D, true, true, true>, k, smem, cls);
      return launch_strips(c, mech_kernel<T, F, E, D, false, true, true>, k, smem, cls);
    }
    if (k.gpm) {  // precomputed Gauss-point moduli: only u is staged
      constexpr int NF = 3;
      const SmemPlan smem{0, (size_t)kRing * NF * 2 * kRowW, 3 * 32, sizeof(T)};
      if (iso(k.g)) return launch_strips(c, mech_kernel<T, F, E, D, true, true>, k, smem, cls);
      return launch_strips(c, mech_kernel<T, F, E, D, false, true>, k, smem, cls);
    }
  }
  constexpr int NF = (D ? 0 : 3) + (F ? 3 : 2);
  const SmemPlan smem{0, (size_t)kRing * NF * 2 * kRowW, 3 * 32, sizeof(T)};
  if constexpr (!D) {
    if (iso(k.g)) return launch_strips(c, mech_kernel<T, F, E, D, true>, k, smem, cls);
  }
  return launch_strips(c, mech_kernel<T, F, E, D, false>, k, smem, cls);
}

static void mech_fields(hpc_ctx* c, int level, bool finest, bool diag, const double* src, MechK& k) {
  const LevelFields& F = c->F[level];
  const LevelGeo& g = c->L[level];
  int f = 0;
  if (!diag)
    for (int m = 0; m < 3; ++m) k.fields[f++] = src + (long long)m * g.n;
  if (finest) {
    k.fields[f++] = F.bulK;
    k.fields[f++] = F.G;
    k.fields[f++] = F.d;
  } else {
    k.fields[f++] = F.Ke;
    k.fields[f++] = F.Ge;
  }
  for (; f < 6; ++f) k.fields[f] = F.bulK;
}

int launch_mech(hpc_ctx* c, const MechCall& m) {
  // the restriction reads the fine residual around each coarse node: a slab takes the neighbours'
  // planes first (SendRecv(rf), multigrid_intergrid.cpp:393)
  if (m.epi == EPI_FAS) HPC_SLAB_HALO(c, m.fine_level, m.rf, 3, sizeof(double));
  MechK k{};
  k.g = c->L[m.level];
  if (m.epi == EPI_FAS) k.gf = c->L[m.fine_level];
  mech_fields(c, m.level, m.finest, false, m.src, k);
  k.out = m.out;
  k.choice = c->F[m.level].choice;
  k.small_k = m.small_k;
  k.fu = m.fu;
  k.set_fnorm = m.set_fnorm;
  k.invM = m.invM;
  k.rf = m.rf;
  k.gpm = (m.finest && c->gpm_active) ? c->F[m.level].gpm : nullptr;
  k.red = make_red(c, m.s_out0, m.s_out1, m.s_out2);
  k.err = c->scal + S_ERR;
  const bool f = m.finest;
  const bool tma = f && k.gpm && c->tma_stage;
  if (tma) {
    const int rc = encode_rows<double>(k.g, k.fields[0], &k.tmap);
    if (rc) return rc;
  }
  switch (m.epi) {
    case EPI_PLAIN: return f ? run_mech<true, EPI_PLAIN, false>(c, k, tma) : run_mech<false, EPI_PLAIN, false>(c, k);
    case EPI_RESIDUAL:
      return f ? run_mech<true, EPI_RESIDUAL, false>(c, k, tma) : run_mech<false, EPI_RESIDUAL, false>(c, k);
    case EPI_PCG: return f ? run_mech<true, EPI_PCG, false>(c, k, tma) : run_mech<false, EPI_PCG, false>(c, k);
    case EPI_FAS: return run_mech<false, EPI_FAS, false>(c, k);
    case EPI_REACTION:
      return f ? run_mech<true, EPI_REACTION, false>(c, k, tma) : run_mech<false, EPI_REACTION, false>(c, k);
  }
  return HPC_ERR_ARG;
}

int launch_mech_diag(hpc_ctx* c, int level, bool finest, double small_k, double* out) {
  MechK k{};
  k.g = c->L[level];
  mech_fields(c, level, finest, true, nullptr, k);
  k.choice = c->F[level].choice;
  k.small_k = small_k;
  k.out = out;
  k.red = make_red(c, -1, -1, -1);
  return finest ? run_mech<true, EPI_PLAIN, true>(c, k) : run_mech<false, EPI_PLAIN, true>(c, k);
}

template <bool F, int E>
static int run_mech_tc(hpc_ctx* c, const MechKT<float>& k) {
  constexpr int NF = 3 + (F ? 0 : 2);
  const SmemPlan smem{(size_t)kTcHead, (size_t)kRing * NF * 2 * kRowW, 3 * 32, sizeof(float)};
  // strip shapes of the latency model (one lockstep block per SM on the large levels); shapes that
  // give every resident block (3 per SM) strips measured slower (MMA round trips share the SM)
  return launch_strips(c, mech_tc_kernel<F, E>, k, smem, (F && E == EPI_PCG) ? HPC_KC_MECH32_PCG_FINEST : HPC_KC_NONE);
}

// Single-precision element operator of the precision form's V-cycle: the same kernels on the FP32
// mirror of a level (LevelF32); residual, PCG apply and FAS right-hand side epilogues.
int launch_mech_f32(hpc_ctx* c, const MechCall32& m) {
  if (m.epi == EPI_FAS) HPC_SLAB_HALO(c, m.fine_level, m.rf, 3, sizeof(float));
  MechKT<float> k{};
  const LevelF32& F = c->F32[m.level];
  const LevelGeo& g = c->L[m.level];
  k.g = g;
  if (m.epi == EPI_FAS) k.gf = c->L[m.fine_level];
  int f = 0;
  for (int q = 0; q < 3; ++q) k.fields[f++] = m.src + (long long)q * g.n;
  if (m.finest) {
    k.fields[f++] = F.K;
    k.fields[f++] = F.G;
    k.fields[f++] = F.d;
  } else {
    k.fields[f++] = F.Ke;
    k.fields[f++] = F.Ge;
  }
  for (; f < 6; ++f) k.fields[f] = k.fields[3];
  k.out = m.out;
  k.choice = c->F[m.level].choice;
  k.small_k = m.small_k;
  k.fu = m.fu;
  k.set_fnorm = 0;
  k.invM = m.invM;
  k.rf = m.rf;
  k.gpm = (m.finest && c->gpm_active) ? F.gpm : nullptr;
  k.red = make_red(c, m.s_out0, m.s_out1, m.s_out2);
  k.err = c->scal + S_ERR;
  const bool fin = m.finest;
  // tensor-core contraction (hpc_set_tensor_apply): isotropic levels, Gauss-point moduli at the finest;
  // not on a slab (its epilogue sums every plane)
  if (c->tc_apply && !c->slab && iso(g) && (!fin || k.gpm)) {
    switch (m.epi) {
      case EPI_PLAIN: return fin ? run_mech_tc<true, EPI_PLAIN>(c, k) : run_mech_tc<false, EPI_PLAIN>(c, k);
      case EPI_RESIDUAL: return fin ? run_mech_tc<true, EPI_RESIDUAL>(c, k) : run_mech_tc<false, EPI_RESIDUAL>(c, k);
      case EPI_PCG: return fin ? run_mech_tc<true, EPI_PCG>(c, k) : run_mech_tc<false, EPI_PCG>(c, k);
      case EPI_FAS: return run_mech_tc<false, EPI_FAS>(c, k);
    }
  }
  const bool tma = fin && k.gpm && c->tma_stage;
  if (tma) {
    const int rc = encode_rows<float>(g, k.fields[0], &k.tmap);
    if (rc) return rc;
  }
  switch (m.epi) {
    case EPI_PLAIN:
      return fin ? run_mech<true, EPI_PLAIN, false>(c, k, tma) : run_mech<false, EPI_PLAIN, false>(c, k);
    case EPI_RESIDUAL:
      return fin ? run_mech<true, EPI_RESIDUAL, false>(c, k, tma) : run_mech<false, EPI_RESIDUAL, false>(c, k);
    case EPI_PCG: return fin ? run_mech<true, EPI_PCG, false>(c, k, tma) : run_mech<false, EPI_PCG, false>(c, k);
    case EPI_FAS: return run_mech<false, EPI_FAS, false>(c, k);
  }
  return HPC_ERR_ARG;
}

// Gauss-point moduli of the finest level, computed once per mechanical solve (the material is
// fixed while the solve runs): the same mech_moduli_finest as the strip kernels, so the applies that
// read them produce the same bits as the applies that interpolate the nodal fields themselves.
template <typename T>
__global__ void gp_material_kernel(LevelGeo g, const T* K, const T* G, const T* d, const int8_t* choice,
                                   double small_k, T* gpm) {
  const SFt<T> s = make_sf<T>(g);
  const bool isotropic = g.hx == g.hy && g.hy == g.hz;
  const T wg = isotropic ? T(g.wg) * (s.ih[0] * s.ih[0]) : T(g.wg);
  const long long ne = (long long)(g.nx - 1) * (g.ny - 1) * (g.nz - 1);
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < ne; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % (g.nx - 1)), j = (int)((q / (g.nx - 1)) % (g.ny - 1)), kz = (int)(q / ((long long)(g.nx - 1) * (g.ny - 1)));
    T Kn[8], Gn[8], dn[8], Kw[8], Gw[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const long long o = nidx(g, i + (n & 1), j + ((n >> 1) & 1), kz + (n >> 2));
      Kn[n] = K[o];
      Gn[n] = G[o];
      dn[n] = d[o];
    }
    const long long e = nidx(g, i, j, kz);
    mech_moduli_finest(Kn, Gn, dn, choice[e], T(small_k), wg, s, Kw, Gw);
#pragma unroll
    for (int q8 = 0; q8 < 8; ++q8) {
      gpm[(long long)q8 * g.n + e] = fma(T(-2.0 / 3.0), Gw[q8], Kw[q8]);  // K - 2G/3
      gpm[(long long)(8 + q8) * g.n + e] = Gw[q8];
    }
  }
}

int launch_gp_material(hpc_ctx* c, double small_k) {
  const int L = c->maxlevel;
  const LevelGeo& g = c->L[L];
  const LevelFields& F = c->F[L];
  const long long ne = (long long)(g.nx - 1) * (g.ny - 1) * (g.nz - 1);
  const int grid = (int)std::min<long long>((ne + 255) / 256, (long long)num_sms() * 8);
  if (grid <= 0) return HPC_OK;
  gp_material_kernel<double><<<grid, 256, 0, c->stream>>>(g, F.bulK, F.G, F.d, F.choice, small_k, F.gpm);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

// ------------------------------------------------------------------------------------------
// phase field
// ------------------------------------------------------------------------------------------
struct PfK {
  LevelGeo g, gf;
  StripGeo sg;
  const double* fields[3];  // staged: x, gc, H (H is element data, read on the lower plane)
  double* out;
  double lc;
  const double* fd;
  const double* invM;
  const double* rf;
  RedTarget red;
};

template <int EPI, bool DIAG, bool ISO>
__global__ void __launch_bounds__(kWarps * 32) pf_kernel(PfK k) {
  constexpr int NF = 3;
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  double* ring = smem + (size_t)wib * (kRing * NF * 2 * kRowW + (k.sg.wy - 1) * 32);
  double* zc = ring + kRing * NF * 2 * kRowW;  // [row][lane]
  const SF s = make_sf(k.g);
  double red0 = 0.0, red1 = 0.0, red2 = 0.0;
  const long long nwarps_total = (long long)gridDim.x * kWarps;
  // ISO: only the gradient term carries 1/h^2 (see sf_forward); the mass term keeps wg
  const double wg = k.g.wg, wgb = ISO ? k.g.wg * (s.ih[0] * s.ih[0]) : k.g.wg, inv_lc = 1.0 / k.lc;
  const double* fptr[NF] = {k.fields[0], k.fields[1], k.fields[2]};

  for (long long strip = (long long)blockIdx.x * kWarps + wib; strip < k.sg.nstrips; strip += nwarps_total) {
    const int sx = (int)(strip % k.sg.tx);
    const long long rest = strip / k.sg.tx;
    const int sy = (int)(rest % k.sg.ty);
    const int sz = (int)(rest / k.sg.ty);
    const int wy = k.sg.wy, rows = wy + 1;
    const int x0 = sx * kOX, y0 = sy * (wy - 1), z0 = sz * k.sg.cz;
    const int x = x0 - 1 + lane;
    const int zend = min(z0 + k.sg.cz - 1, k.g.nz - 1);
    Stream<NF> st{ring, fptr, x, y0, z0, zend - z0 + 2, 0, rows, &k.g};
    st.total = st.nlayers * rows;
    st.issue(0, lane);
    st.issue(1, lane);
    double yp[2] = {0.0, 0.0};
    for (int si = 0; si < st.total; ++si) {
      st.issue(si + 2, lane);
      cp_async_wait2();
      __syncwarp();
      const int li = si / rows, r = si - li * rows;
      const int kk = z0 - 1 + li;
      if (r == 0) {
        yp[0] = yp[1] = 0.0;
        __syncwarp();
        continue;
      }
      const int rr = r - 1, ey = y0 - 1 + rr;
      double f[8];
      const bool valid = lane < 31 && x >= 0 && x <= k.g.nx - 2 && ey >= 0 && ey <= k.g.ny - 2 && kk >= 0 &&
                         kk <= k.g.nz - 2;
      if (valid) {
        double gcn[8], gcg[8], aw[8], bw[8];
#pragma unroll
        for (int n = 0; n < 8; ++n) {
          const int a = n & 1, b = (n >> 1) & 1, c = n >> 2;
          gcn[n] = st.at(b ? si : si - 1, 1, c, lane + a);
        }
        gp_material(gcn, s, gcg);
        const double H2 = 2.0 * st.at(si - 1, 2, 0, lane);
#pragma unroll
        for (int g = 0; g < 8; ++g) {
          aw[g] = wg * fma(gcg[g], inv_lc, H2);
          bw[g] = wgb * (gcg[g] * k.lc);
        }
        if (DIAG) {
          pf_element_diag(aw, bw, s, f);
        } else {
          double xv[8];
#pragma unroll
          for (int n = 0; n < 8; ++n) {
            const int a = n & 1, b = (n >> 1) & 1, c = n >> 2;
            xv[n] = st.at(b ? si : si - 1, 0, c, lane + a);
          }
          pf_element<ISO>(xv, aw, bw, s, f);
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
            const bool own = owned_plane(k.g, kk);
            const double s0 = fma(fv, fv, red0), s1 = fma(rv, rv, red1);
            red0 = own ? s0 : red0;
            red1 = own ? s1 : red1;
            if (k.invM) {
              const double s2 = fma(rv, rv * k.invM[n], red2);
              red2 = own ? s2 : red2;
            }
          } else if (EPI == EPI_PCG) {
            k.out[n] = tot;
            const double s0 = fma(st.at(si - 1, 0, 0, lane), tot, red0);
            red0 = owned_plane(k.g, kk) ? s0 : red0;
          } else if (EPI == EPI_FAS) {
            const int fz = 2 * kk + k.g.zsh;
            k.out[n] = tot + (fz >= 0 ? full_weight(k.gf, k.rf, 2 * x, 2 * ey, fz) : 0.0);
          }
        }
      }
      yp[0] = X[1][0];
      yp[1] = X[1][1];
      __syncwarp();
    }
  }
  if (EPI == EPI_RESIDUAL || EPI == EPI_PCG) {
    double v[3] = {red0, red1, red2};
    grid_reduce<3>(v, k.red);
  }
}

template <int E, bool D>
static int run_pf(hpc_ctx* c, const PfK& k, bool finest) {
  const SmemPlan smem{0, (size_t)kRing * 3 * 2 * kRowW, 32, sizeof(double)};
  const int cls = (finest && E == EPI_PCG && !D) ? HPC_KC_PF_PCG_FINEST : HPC_KC_NONE;
  if constexpr (!D) {
    if (iso(k.g)) return launch_strips(c, pf_kernel<E, D, true>, k, smem, cls);
  }
  return launch_strips(c, pf_kernel<E, D, false>, k, smem, cls);
}

int launch_pf(hpc_ctx* c, const PfCall& p) {
  if (p.epi == EPI_FAS) HPC_SLAB_HALO(c, p.fine_level, p.rf, 1, sizeof(double));  // SendRecv(rf), :356
  PfK k{};
  k.g = c->L[p.level];
  if (p.epi == EPI_FAS) k.gf = c->L[p.fine_level];
  k.fields[0] = p.src;
  k.fields[1] = c->F[p.level].gc;
  k.fields[2] = c->F[p.level].H;
  k.out = p.out;
  k.lc = p.lc;
  k.fd = p.fd;
  k.invM = p.invM;
  k.rf = p.rf;
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
  k.fields[0] = c->F[level].d;
  k.fields[1] = c->F[level].gc;
  k.fields[2] = c->F[level].H;
  k.out = out;
  k.lc = lc;
  k.red = make_red(c, -1, -1, -1);
  return run_pf<EPI_PLAIN, true>(c, k, false);
}

}  // namespace hpc
