// Device helpers shared by the kernels: deterministic reductions, Dirichlet flags, and the
// sum-factorised trilinear (Q1, 2x2x2 Gauss) element algebra.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "internal.h"

namespace hpc {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

enum RedOp { RED_SUM = 0, RED_MAX = 1, RED_MIN = 2 };

template <int OP>
__device__ __forceinline__ double red_combine(double a, double b) {
  if (OP == RED_SUM) return a + b;
  if (OP == RED_MAX) return fmax(a, b);
  return fmin(a, b);
}
template <int OP>
__device__ __forceinline__ double warp_red(double v) {
  if (OP == RED_SUM) return warp_sum(v);
  if (OP == RED_MAX) return warp_max(v);
  return warp_min(v);
}
template <int OP>
__device__ __forceinline__ double red_identity() {
  if (OP == RED_SUM) return 0.0;
  if (OP == RED_MAX) return -1.0 / 0.0;
  return 1.0 / 0.0;
}

struct RedTarget {
  double* partials;      // >= NR * gridDim.x doubles
  unsigned int* counter; // zero between kernels
  double* scal;          // scalar pool
  int slot[3];           // destination slots (-1 = discard)
};
// The reduction target of a context for the next launch; on a z-slab context the slots are also
// recorded so that the launch check combines them over the ranks with `op` (a RedOp).
RedTarget make_red(hpc_ctx* c, int s0, int s1, int s2, int op = RED_SUM);

// Block-wide reduction of NR values per thread followed by a deterministic grid-wide
// combination: every block stores its partials; the last block to finish combines them in
// block order (fixed strided pattern + fixed shuffle tree), so the result does not depend on
// block scheduling.  Must be called by every thread of every block (1-D grid, blockDim.x a
// multiple of 32, at most 1024).
template <int NR, int OP = RED_SUM>
__device__ void grid_reduce(double (&v)[NR], const RedTarget& t) {
  __shared__ double sred[NR][32];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int nb = gridDim.x;
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    double x = warp_red<OP>(v[r]);
    if (lane == 0) sred[r][warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      double x = lane < nwarps ? sred[r][lane] : red_identity<OP>();
      x = warp_red<OP>(x);
      if (lane == 0) t.partials[(size_t)r * nb + blockIdx.x] = x;
    }
    if (lane == 0) {
      __threadfence();
      unsigned prev = atomicAdd(t.counter, 1u);
      s_last = (prev == (unsigned)nb - 1u);
    }
  }
  __syncthreads();
  if (s_last && warp == 0) {
    __threadfence();
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      double x = red_identity<OP>();
      for (int i = lane; i < nb; i += 32) x = red_combine<OP>(x, __ldcg(t.partials + (size_t)r * nb + i));
      x = warp_red<OP>(x);
      if (lane == 0 && t.slot[r] >= 0) t.scal[t.slot[r]] = x;
    }
    if (lane == 0) *t.counter = 0u;
  }
}

// A z plane this rank owns: reductions sum over owned nodes only (realdomain, pcg_utilities.cpp:16-58);
// every plane of a whole specimen.
__device__ __forceinline__ bool owned_plane(const LevelGeo& g, int k) { return k >= g.oz0 && k < g.oz1; }

// Dirichlet node sets of boundary_conditions.cpp:20-154 from the separable axis flags.
struct BcFlags {
  bool c0, c1, c2, top;
};
__device__ __forceinline__ BcFlags bc_flags(const LevelGeo& g, int i, int j, int k) {
  const uint8_t fx = g.bx[i], fy = g.by[j], fz = g.bz[k];
  BcFlags b;
  b.c0 = (fz & 1) && (fx & 1) && (fy & 1);  // z == za && x == (xa+xb)/2 && y == ya
  b.c1 = (fz & 1) && (fx & 2) && (fy & 2);  // z == za && x == xb && y == (ya+yb)/2
  b.c2 = (fz & 3) != 0;                     // z == za || z == zb
  b.top = (fz & 2) != 0;                    // z == zb (the later assignment wins: Ut)
  return b;
}

// ---------------------------------------------------------------------------------------------
// Sum-factorised Q1 algebra.  Element nodes are numbered lexicographically n = a + 2b + 4c for the
// node at offset (a,b,c); Gauss points likewise g = q + 2p + 4r at local coordinates
// (t[q], t[p], t[r]) in [0,1], t = (1 -+ 1/sqrt 3)/2.  The 1-D shape values at a Gauss point are
// 1 - t and t, the 1-D derivative is (u1 - u0)/h, as in Dshape_function (shape_function.cpp:16-75).
// Every Gauss point carries the same weight wg = hx*hy*hz/8, which callers fold into the material.
// ---------------------------------------------------------------------------------------------
template <typename T>
struct SFt {
  T t[2];
  T ih[3];  // 1/hx, 1/hy, 1/hz
};
using SF = SFt<double>;

// x == +-0 from the bit pattern (integer pipe); v exactly zero is what gauss_point_MP tests.
__device__ __forceinline__ bool bits_zero(double v) { return (__double_as_longlong(v) << 1) == 0; }
__device__ __forceinline__ bool bits_zero(float v) { return (__float_as_uint(v) << 1) == 0u; }

// Gradient of a trilinear field at the 8 Gauss points.  d/dx is independent of the x Gauss index,
// so it has 4 distinct values gx[p + 2r]; likewise gy[q + 2r], gz[q + 2p].  Optionally the values
// at the Gauss points, val[q + 2p + 4r].  ISO (hx = hy = hz): the gradients are left unscaled by
// 1/h; callers fold 1/h^2 into the material, which is exact when h is a power of two (every level
// of a hierarchy whose finest spacing is 1, as the reference's voxel domains have).
template <bool ISO = false, typename T>
__device__ __forceinline__ void sf_forward(const T (&u)[8], const SFt<T>& s, T (&gx)[4], T (&gy)[4], T (&gz)[4],
                                           T* val) {
  T dx[4], ix[2][4], dy[2][2];
#pragma unroll
  for (int bc = 0; bc < 4; ++bc) dx[bc] = u[2 * bc + 1] - u[2 * bc];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int bc = 0; bc < 4; ++bc) ix[q][bc] = fma(s.t[q], dx[bc], u[2 * bc]);
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int c = 0; c < 2; ++c) dy[q][c] = ix[q][1 + 2 * c] - ix[q][2 * c];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const T i0 = fma(s.t[p], dy[q][0], ix[q][0]);
      const T i1 = fma(s.t[p], dy[q][1], ix[q][2]);
      const T dz = i1 - i0;
      gz[q + 2 * p] = ISO ? dz : dz * s.ih[2];
      if (val) {
        val[q + 2 * p] = fma(s.t[0], dz, i0);
        val[q + 2 * p + 4] = fma(s.t[1], dz, i0);
      }
    }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const T e = dy[q][1] - dy[q][0];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const T v = fma(s.t[r], e, dy[q][0]);
      gy[q + 2 * r] = ISO ? v : v * s.ih[1];
    }
  }
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const T e0 = fma(s.t[p], dx[1] - dx[0], dx[0]);
    const T e1 = fma(s.t[p], dx[3] - dx[2], dx[2]);
    const T e = e1 - e0;
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const T v = fma(s.t[r], e, e0);
      gx[p + 2 * r] = ISO ? v : v * s.ih[0];
    }
  }
}

// Exact transpose of sf_forward: given adjoints of gx, gy, gz (and optionally of the Gauss-point
// values), accumulates the nodal adjoint f[8] (f is overwritten).
template <bool ISO = false, typename T>
__device__ __forceinline__ void sf_adjoint(const T (&sgx)[4], const T (&sgy)[4], const T (&sgz)[4], const T* sval,
                                           const SFt<T>& s, T (&f)[8]) {
  const T t0 = s.t[0], t1 = s.t[1], u0 = T(1) - t0, u1 = T(1) - t1;
  // gx[p+2r] = ih0 * ((1-t_r) ey[p][0] + t_r ey[p][1]);  ey[p][c] = (1-t_p) dx[2c] + t_p dx[2c+1]
  T Adx[4];
  {
    const T ihx = s.ih[0];
    const T a00 = ISO ? sgx[0] : sgx[0] * ihx, a10 = ISO ? sgx[1] : sgx[1] * ihx;
    const T a01 = ISO ? sgx[2] : sgx[2] * ihx, a11 = ISO ? sgx[3] : sgx[3] * ihx;
    // Aey[p][c]
    const T e00 = u0 * a00 + u1 * a01, e01 = t0 * a00 + t1 * a01;  // p = 0
    const T e10 = u0 * a10 + u1 * a11, e11 = t0 * a10 + t1 * a11;  // p = 1
    Adx[0] = u0 * e00 + u1 * e10;
    Adx[1] = t0 * e00 + t1 * e10;
    Adx[2] = u0 * e01 + u1 * e11;
    Adx[3] = t0 * e01 + t1 * e11;
  }
  // gy[q+2r] = ih1 * ((1-t_r) dy[q][0] + t_r dy[q][1])
  T Ady[2][2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const T a0 = ISO ? sgy[q] : sgy[q] * s.ih[1], a1 = ISO ? sgy[q + 2] : sgy[q + 2] * s.ih[1];
    Ady[q][0] = u0 * a0 + u1 * a1;
    Ady[q][1] = t0 * a0 + t1 * a1;
  }
  // gz[q+2p] = ih2 * (iy[q][p][1] - iy[q][p][0]);  val = iy[q][p][0] + t_r (iy[..][1] - iy[..][0])
  T Aiy[2][2][2];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      T adz = ISO ? sgz[q + 2 * p] : sgz[q + 2 * p] * s.ih[2];
      T a0 = T(0);
      if (sval) {
        const T v0 = sval[q + 2 * p], v1 = sval[q + 2 * p + 4];
        adz += t0 * v0 + t1 * v1;
        a0 = v0 + v1;
      }
      Aiy[q][p][1] = adz;
      Aiy[q][p][0] = a0 - adz;
    }
  // iy[q][p][c] = ix[q][2c] + t_p dy[q][c];  dy[q][c] = ix[q][2c+1] - ix[q][2c]
  T Aix[2][4];
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const T s0 = Aiy[q][0][c] + Aiy[q][1][c];
      const T ady = Ady[q][c] + t0 * Aiy[q][0][c] + t1 * Aiy[q][1][c];
      Aix[q][2 * c + 1] = ady;
      Aix[q][2 * c] = s0 - ady;
    }
  // ix[q][bc] = u[2bc] + t_q dx[bc];  dx[bc] = u[2bc+1] - u[2bc]
#pragma unroll
  for (int bc = 0; bc < 4; ++bc) {
    const T adx = Adx[bc] + t0 * Aix[0][bc] + t1 * Aix[1][bc];
    f[2 * bc + 1] = adx;
    f[2 * bc] = Aix[0][bc] + Aix[1][bc] - adx;
  }
}

// Trilinear values of a nodal field at the 8 Gauss points.
template <typename T>
__device__ __forceinline__ void sf_interp(const T (&v)[8], const SFt<T>& s, T (&out)[8]) {
  T ix[2][4];
#pragma unroll
  for (int bc = 0; bc < 4; ++bc) {
    const T d = v[2 * bc + 1] - v[2 * bc];
    ix[0][bc] = fma(s.t[0], d, v[2 * bc]);
    ix[1][bc] = fma(s.t[1], d, v[2 * bc]);
  }
#pragma unroll
  for (int q = 0; q < 2; ++q)
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      const T i0 = fma(s.t[p], ix[q][1] - ix[q][0], ix[q][0]);
      const T i1 = fma(s.t[p], ix[q][3] - ix[q][2], ix[q][2]);
      const T dz = i1 - i0;
      out[q + 2 * p] = fma(s.t[0], dz, i0);
      out[q + 2 * p + 4] = fma(s.t[1], dz, i0);
    }
}

// gauss_point_MP (material_gauss_point.cpp:18-41): 0 at every Gauss point if any nodal value is
// exactly 0, else the trilinear values.
template <typename T>
__device__ __forceinline__ void gp_material(const T (&v)[8], const SFt<T>& s, T (&out)[8]) {
  bool zero = false;  // v == +-0, tested on the bit pattern (integer pipe, not the floating-point unit)
#pragma unroll
  for (int n = 0; n < 8; ++n) zero |= bits_zero(v[n]);
  if (zero) {
#pragma unroll
    for (int g = 0; g < 8; ++g) out[g] = T(0);
  } else {
    sf_interp(v, s, out);
  }
}

// Element stiffness action K_e u_e for Q1 small-strain elasticity with per-Gauss-point moduli
// (Internal_Force_element, mechanical_pcg.cpp:114-172): sigma = K tr(eps) I + 2G dev(eps).
// Kw, Gw already include the Gauss weight wg.
// LAM: Kw holds the first Lame coefficient K - 2G/3 (times wg) instead of K, as the precomputed
// Gauss-point moduli store it (the same fma, done once per solve instead of in every apply).
template <bool ISO = false, typename T, bool LAM = false>
__device__ __forceinline__ void mech_element(const T (&u)[3][8], const T (&Kw)[8], const T (&Gw)[8],
                                             const SFt<T>& s, T (&f)[3][8]) {
  T gx[3][4], gy[3][4], gz[3][4];
#pragma unroll
  for (int m = 0; m < 3; ++m) sf_forward<ISO>(u[m], s, gx[m], gy[m], gz[m], (T*)nullptr);
  T sx[3][4], sy[3][4], sz[3][4];
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int i = 0; i < 4; ++i) sx[m][i] = sy[m][i] = sz[m][i] = T(0);
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int g = q + 2 * p + 4 * r, ix = p + 2 * r, iy = q + 2 * r, iz = q + 2 * p;
        const T exx = gx[0][ix], eyy = gy[1][iy], ezz = gz[2][iz];
        const T gxy = gx[1][ix] + gy[0][iy];
        const T gxz = gx[2][ix] + gz[0][iz];
        const T gyz = gy[2][iy] + gz[1][iz];
        const T K = Kw[g], G = Gw[g];
        const T tr = exx + eyy + ezz;
        const T lt = (LAM ? K : fma(T(-2.0 / 3.0), G, K)) * tr;
        const T G2 = G + G;
        const T sxx = fma(G2, exx, lt), syy = fma(G2, eyy, lt), szz = fma(G2, ezz, lt);
        const T sxy = G * gxy, sxz = G * gxz, syz = G * gyz;
        sx[0][ix] += sxx; sx[1][ix] += sxy; sx[2][ix] += sxz;
        sy[0][iy] += sxy; sy[1][iy] += syy; sy[2][iy] += syz;
        sz[0][iz] += sxz; sz[1][iz] += syz; sz[2][iz] += szz;
      }
#pragma unroll
  for (int m = 0; m < 3; ++m) sf_adjoint<ISO>(sx[m], sy[m], sz[m], (const T*)nullptr, s, f[m]);
}

// Diagonal of the element stiffness (PreM_u_element, mechanical_pcg.cpp:63-100):
//   diag_x(n) = sum_g wg [(K + 4G/3) dNx^2 + G (dNy^2 + dNz^2)], etc.
__device__ __forceinline__ void mech_element_diag(const double (&Kw)[8], const double (&Gw)[8], const SF& s,
                                                  double (&f)[3][8]) {
  // squared 1-D shape values at Gauss point q for node offset a: w2[a][q]
  const double w2[2][2] = {{(1.0 - s.t[0]) * (1.0 - s.t[0]), (1.0 - s.t[1]) * (1.0 - s.t[1])},
                           {s.t[0] * s.t[0], s.t[1] * s.t[1]}};
  double A[8];
#pragma unroll
  for (int g = 0; g < 8; ++g) A[g] = fma(4.0 / 3.0, Gw[g], Kw[g]);
  // projections P_yz[W](b,c) = sum_g W_g w2[b][p] w2[c][r], etc.
  auto proj = [&](const double (&W)[8], int dir, int i0, int i1) -> double {
    double acc = 0.0;
#pragma unroll
    for (int g = 0; g < 8; ++g) {
      const int q = g & 1, p = (g >> 1) & 1, r = g >> 2;
      double w;
      if (dir == 0) w = w2[i0][p] * w2[i1][r];
      else if (dir == 1) w = w2[i0][q] * w2[i1][r];
      else w = w2[i0][q] * w2[i1][p];
      acc = fma(W[g], w, acc);
    }
    return acc;
  };
  const double ihx2 = s.ih[0] * s.ih[0], ihy2 = s.ih[1] * s.ih[1], ihz2 = s.ih[2] * s.ih[2];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const int a = n & 1, b = (n >> 1) & 1, c = n >> 2;
    const double Ayz = proj(A, 0, b, c), Axz = proj(A, 1, a, c), Axy = proj(A, 2, a, b);
    const double Byz = proj(Gw, 0, b, c), Bxz = proj(Gw, 1, a, c), Bxy = proj(Gw, 2, a, b);
    f[0][n] = Ayz * ihx2 + Bxz * ihy2 + Bxy * ihz2;
    f[1][n] = Byz * ihx2 + Axz * ihy2 + Bxy * ihz2;
    f[2][n] = Byz * ihx2 + Bxz * ihy2 + Axy * ihz2;
  }
}

// Phase-field element action (Fld_element, phase_field_pcg.cpp:61-91):
//   f_sf = sum_g [aw_g N_sf x_g + bw_g dN_sf . dx_g],  aw = wg (2H + gc_g/lc), bw = wg gc_g lc.
template <bool ISO = false>
__device__ __forceinline__ void pf_element(const double (&x)[8], const double (&aw)[8], const double (&bw)[8],
                                           const SF& s, double (&f)[8]) {
  double gx[4], gy[4], gz[4], val[8];
  sf_forward<ISO>(x, s, gx, gy, gz, val);
  double sgx[4] = {0, 0, 0, 0}, sgy[4] = {0, 0, 0, 0}, sgz[4] = {0, 0, 0, 0}, sv[8];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int g = q + 2 * p + 4 * r;
        sv[g] = aw[g] * val[g];
        sgx[p + 2 * r] = fma(bw[g], gx[p + 2 * r], sgx[p + 2 * r]);
        sgy[q + 2 * r] = fma(bw[g], gy[q + 2 * r], sgy[q + 2 * r]);
        sgz[q + 2 * p] = fma(bw[g], gz[q + 2 * p], sgz[q + 2 * p]);
      }
  sf_adjoint<ISO>(sgx, sgy, sgz, sv, s, f);
}

// Diagonal of the phase-field element matrix (Md_element, phase_field_pcg.cpp:20-47).
__device__ __forceinline__ void pf_element_diag(const double (&aw)[8], const double (&bw)[8], const SF& s,
                                                double (&f)[8]) {
  const double w2[2][2] = {{(1.0 - s.t[0]) * (1.0 - s.t[0]), (1.0 - s.t[1]) * (1.0 - s.t[1])},
                           {s.t[0] * s.t[0], s.t[1] * s.t[1]}};
  const double ihx2 = s.ih[0] * s.ih[0], ihy2 = s.ih[1] * s.ih[1], ihz2 = s.ih[2] * s.ih[2];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const int a = n & 1, b = (n >> 1) & 1, c = n >> 2;
    double acc = 0.0;
#pragma unroll
    for (int g = 0; g < 8; ++g) {
      const int q = g & 1, p = (g >> 1) & 1, r = g >> 2;
      const double nx2 = w2[a][q], ny2 = w2[b][p], nz2 = w2[c][r];
      const double grad2 = ny2 * nz2 * ihx2 + nx2 * nz2 * ihy2 + nx2 * ny2 * ihz2;
      acc = fma(aw[g], nx2 * ny2 * nz2, acc);
      acc = fma(bw[g], grad2, acc);
    }
    f[n] = acc;
  }
}

// Strain tensor at a Gauss point from the gradients (symmetric part).
struct Strain {
  double xx, yy, zz, xy, xz, yz;  // tensor components (xy = eps_xy)
};
__device__ __forceinline__ Strain strain_at(const double (&gx)[3][4], const double (&gy)[3][4],
                                            const double (&gz)[3][4], int q, int p, int r) {
  const int ix = p + 2 * r, iy = q + 2 * r, iz = q + 2 * p;
  Strain e;
  e.xx = gx[0][ix];
  e.yy = gy[1][iy];
  e.zz = gz[2][iz];
  e.xy = 0.5 * (gx[1][ix] + gy[0][iy]);
  e.xz = 0.5 * (gx[2][ix] + gz[0][iz]);
  e.yz = 0.5 * (gy[2][iy] + gz[1][iz]);
  return e;
}
// Phi_positive / Phi_negative (strain_history.cpp:134-159) with epsilon_dev (mechanical_strain.cpp:47-61).
__device__ __forceinline__ double eps_dev2(const Strain& e) {
  const double third = (1.0 / 3.0) * (e.xx + e.yy + e.zz);
  const double a = e.xx - third, b = e.yy - third, c = e.zz - third;
  return a * a + b * b + c * c + 2.0 * (e.xy * e.xy + e.xz * e.xz + e.yz * e.yz);
}
__device__ __forceinline__ double phi_pos(double K, double G, const Strain& e) {
  const double tr = e.xx + e.yy + e.zz;
  const double dd = eps_dev2(e);
  return tr >= 0 ? 0.5 * K * tr * tr + G * dd : G * dd;
}
__device__ __forceinline__ double phi_neg(double K, const Strain& e) {
  const double tr = e.xx + e.yy + e.zz;
  return tr >= 0 ? 0.0 : 0.5 * K * tr * tr;
}

template <typename T = double>
__device__ __forceinline__ SFt<T> make_sf(const LevelGeo& g) {
  SFt<T> s;
  const double r3 = 0.57735026918962584;  // 1/sqrt(3)
  s.t[0] = T(0.5 * (1.0 - r3));
  s.t[1] = T(0.5 * (1.0 + r3));
  s.ih[0] = T(1.0 / g.hx);
  s.ih[1] = T(1.0 / g.hy);
  s.ih[2] = T(1.0 / g.hz);
  return s;
}

// Whether the reference's MP_choice loop (material_selection.cpp:59-63) reaches flat slot b of an
// nx*ny*nz level: that loop runs i over the y extent and j over the x extent, and every access is a
// flat offset from b = i + j*nx + k*nx*ny.  For nx == ny this is every element.
__device__ __host__ __forceinline__ bool choice_in_image(long long b, long long nx, long long ny, long long nz) {
  const long long P = nx * ny, z = b / P, rmax = (ny - 2) + (nx - 2) * nx;
  for (long long kp = (z < nz - 2 ? z : nz - 2); kp >= 0; --kp) {
    const long long r = b - kp * P;
    if (r > rmax) break;
    const long long jlo = r - (ny - 2) <= 0 ? 0 : (r - (ny - 2) + nx - 1) / nx;
    const long long jhi = r / nx < nx - 2 ? r / nx : nx - 2;
    if (jlo <= jhi) return true;
  }
  return false;
}

__device__ __forceinline__ long long nidx(const LevelGeo& g, int i, int j, int k) {
  return (long long)i + (long long)j * g.px + (long long)k * g.plane;
}

// Full-weighting restriction of a fine residual at coarse node (fx/2, fy/2, fz/2), neighbours outside
// the fine grid counted as 0, in the reference's term order (multigrid_intergrid.cpp:124-342).
template <typename T>
__device__ __forceinline__ T full_weight(const LevelGeo& gf, const T* rf, int fx, int fy, int fz) {
  const int Xl = gf.nx - 2, Yl = gf.ny - 2, Zl = gf.nz - 2;
  auto R = [&](int a, int b, int c) -> T { return rf[nidx(gf, a, b, c)]; };
  const bool xm = fx < 1, xp = fx > Xl, ym = fy < 1, yq = fy > Yl, zm = fz < 1, zq = fz > Zl;
  const T r11 = (xm || ym || zm) ? T(0) : R(fx - 1, fy - 1, fz - 1);
  const T r12 = (xm || ym || zq) ? T(0) : R(fx - 1, fy - 1, fz + 1);
  const T r13 = (xm || yq || zm) ? T(0) : R(fx - 1, fy + 1, fz - 1);
  const T r14 = (xm || yq || zq) ? T(0) : R(fx - 1, fy + 1, fz + 1);
  const T r15 = (xp || ym || zm) ? T(0) : R(fx + 1, fy - 1, fz - 1);
  const T r16 = (xp || ym || zq) ? T(0) : R(fx + 1, fy - 1, fz + 1);
  const T r17 = (xp || yq || zm) ? T(0) : R(fx + 1, fy + 1, fz - 1);
  const T r18 = (xp || yq || zq) ? T(0) : R(fx + 1, fy + 1, fz + 1);
  const T r21 = (xm || ym) ? T(0) : R(fx - 1, fy - 1, fz);
  const T r22 = (xm || yq) ? T(0) : R(fx - 1, fy + 1, fz);
  const T r23 = (xp || ym) ? T(0) : R(fx + 1, fy - 1, fz);
  const T r24 = (xp || yq) ? T(0) : R(fx + 1, fy + 1, fz);
  const T r25 = (xm || zm) ? T(0) : R(fx - 1, fy, fz - 1);
  const T r26 = (xm || zq) ? T(0) : R(fx - 1, fy, fz + 1);
  const T r27 = (xp || zm) ? T(0) : R(fx + 1, fy, fz - 1);
  const T r28 = (xp || zq) ? T(0) : R(fx + 1, fy, fz + 1);
  const T r29 = (ym || zm) ? T(0) : R(fx, fy - 1, fz - 1);
  const T r210 = (ym || zq) ? T(0) : R(fx, fy - 1, fz + 1);
  const T r211 = (yq || zm) ? T(0) : R(fx, fy + 1, fz - 1);
  const T r212 = (yq || zq) ? T(0) : R(fx, fy + 1, fz + 1);
  const T r41 = zm ? T(0) : R(fx, fy, fz - 1);
  const T r42 = zq ? T(0) : R(fx, fy, fz + 1);
  const T r43 = ym ? T(0) : R(fx, fy - 1, fz);
  const T r44 = yq ? T(0) : R(fx, fy + 1, fz);
  const T r45 = xm ? T(0) : R(fx - 1, fy, fz);
  const T r46 = xp ? T(0) : R(fx + 1, fy, fz);
  const T r8 = R(fx, fy, fz);
  const T s8 = r11 + r12 + r13 + r14 + r15 + r16 + r17 + r18;
  const T s12 = r21 + r22 + r23 + r24 + r25 + r26 + r27 + r28 + r29 + r210 + r211 + r212;
  const T s6 = r41 + r42 + r43 + r44 + r45 + r46;
  return T(0.125) * (s8 + T(2) * s12 + T(4) * s6 + T(8) * r8);
}

}  // namespace hpc
