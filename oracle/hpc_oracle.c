/*
 * hpc_oracle.c - plain-C restatement of the HPCrack hot path (TEST ORACLE).
 *
 * Test infrastructure only: the CUDA library is checked against these
 * functions; the product never links or calls them.  Each function restates
 * the reference routine it cites (path:line inside the HPCrack project), in
 * the same arithmetic order, so that the only differences from the reference
 * are the summation order of the element scatter (the reference scatters in a
 * thread-dependent order under `omp critical`; here element layers of one
 * parity run in parallel, which is deterministic) and the order of the global
 * sums.  Parity with the reference itself is pinned by tests/golden/.
 */
#include "hpc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const int CX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
static const int CY[8] = {0, 0, 1, 1, 0, 0, 1, 1};
static const int CZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};

/* ------------------------------------------------------------------------- */
/* geometry                                                                  */
/* ------------------------------------------------------------------------- */

/* input_setting (image_input.cpp:21-27) + initialize (initialization.cpp:19-134), one rank. */
void orc_geom_init(orc_geom* g, int maxlevel, const int* enb, const double* x0, const int* roi) {
  memset(g, 0, sizeof *g);
  g->maxlevel = maxlevel;
  for (int a = 0; a < 3; ++a) {
    g->enb[a] = enb[a];
    g->roi[a] = roi[a];
    g->x0[a] = x0[a];
  }
  int coefb[3];
  for (int a = 0; a < 3; ++a) coefb[a] = roi[a] + enb[a] * (int)pow(2, maxlevel);
  g->box[0] = x0[0];
  g->box[1] = x0[0] + coefb[0];
  g->box[2] = x0[1];
  g->box[3] = x0[1] + coefb[1];
  g->box[4] = x0[2];
  g->box[5] = x0[2] + coefb[2];
  double hx = (g->box[1] - g->box[0]) / enb[0];
  double hy = (g->box[3] - g->box[2]) / enb[1];
  double hz = (g->box[5] - g->box[4]) / enb[2];
  int nx = enb[0] + 1, ny = enb[1] + 1, nz = enb[2] + 1;
  for (int l = 0; l <= maxlevel; ++l) {
    g->lv[l].nx = nx;
    g->lv[l].ny = ny;
    g->lv[l].nz = nz;
    g->lv[l].hx = hx;
    g->lv[l].hy = hy;
    g->lv[l].hz = hz;
    hx *= 0.5;
    hy *= 0.5;
    hz *= 0.5;
    nx = 2 * (nx - 1) + 1;
    ny = 2 * (ny - 1) + 1;
    nz = 2 * (nz - 1) + 1;
  }
}

static long lvl_n(const orc_lvl* L) { return (long)L->nx * L->ny * L->nz; }

/* ------------------------------------------------------------------------- */
/* shape functions (shape_function.cpp:16-75)                                */
/* ------------------------------------------------------------------------- */

typedef struct {
  double N[8][8];      /* N(g, n) */
  double DN[3][8][8];  /* DN(c, g, n) */
  double wg;
} shp;

static void shape_init(shp* s, double hx, double hy, double hz) {
  double x[8] = {-1., 1., 1., -1., -1., 1., 1., -1.};
  double y[8] = {-1., -1., 1., 1., -1., -1., 1., 1.};
  double z[8] = {-1., -1., -1., -1., 1., 1., 1., 1.};
  double w[8];
  double x1 = 0, x2 = 0, y1 = 0, y2 = 0, z1 = 0, z2 = 0, detJ = 0;
  for (int i = 0; i < 8; i++) {
    x[i] = x[i] / sqrt(3);
    y[i] = y[i] / sqrt(3);
    z[i] = z[i] / sqrt(3);
    s->N[i][0] = 0.125 * (1 - x[i]) * (1 - y[i]) * (1 - z[i]);
    s->N[i][1] = 0.125 * (1 + x[i]) * (1 - y[i]) * (1 - z[i]);
    s->N[i][2] = 0.125 * (1 + x[i]) * (1 + y[i]) * (1 - z[i]);
    s->N[i][3] = 0.125 * (1 - x[i]) * (1 + y[i]) * (1 - z[i]);
    s->N[i][4] = 0.125 * (1 - x[i]) * (1 - y[i]) * (1 + z[i]);
    s->N[i][5] = 0.125 * (1 + x[i]) * (1 - y[i]) * (1 + z[i]);
    s->N[i][6] = 0.125 * (1 + x[i]) * (1 + y[i]) * (1 + z[i]);
    s->N[i][7] = 0.125 * (1 - x[i]) * (1 + y[i]) * (1 + z[i]);
    for (int c = 0; c < 3; c++) {
      if (c == 0) { x1 = 2; x2 = 0; y1 = y[i]; y2 = y[i]; z1 = z[i]; z2 = z[i]; detJ = 2. / hx; }
      if (c == 1) { x1 = x[i]; x2 = x[i]; y1 = 2; y2 = 0; z1 = z[i]; z2 = z[i]; detJ = 2. / hy; }
      if (c == 2) { x1 = x[i]; x2 = x[i]; y1 = y[i]; y2 = y[i]; z1 = 2; z2 = 0; detJ = 2. / hz; }
      w[0] = 0.125 * (1 - x1) * (1 - y1) * (1 - z1);
      w[1] = 0.125 * (1 + x2) * (1 - y1) * (1 - z1);
      w[2] = 0.125 * (1 + x2) * (1 + y2) * (1 - z1);
      w[3] = 0.125 * (1 - x1) * (1 + y2) * (1 - z1);
      w[4] = 0.125 * (1 - x1) * (1 - y1) * (1 + z2);
      w[5] = 0.125 * (1 + x2) * (1 - y1) * (1 + z2);
      w[6] = 0.125 * (1 + x2) * (1 + y2) * (1 + z2);
      w[7] = 0.125 * (1 - x1) * (1 + y2) * (1 + z2);
      for (int j = 0; j < 8; j++) s->DN[c][i][j] = w[j] * detJ;
    }
  }
  s->wg = 0.125 * hx * hy * hz;
}

static void node_offsets(const orc_lvl* L, long off[8]) {
  long sx = 1, sy = L->nx, sz = (long)L->nx * L->ny;
  for (int n = 0; n < 8; ++n) off[n] = CX[n] * sx + CY[n] * sy + CZ[n] * sz;
}

/* ------------------------------------------------------------------------- */
/* Gauss-point material (material_gauss_point.cpp:18-59)                     */
/* ------------------------------------------------------------------------- */

/* gauss_point_MP: 0 if any of the 8 nodal values is exactly 0, else the trilinear value. */
static double gpmp(const double* MP, long e, const long off[8], const double* Ng) {
  int a = 1;
  for (int n = 0; n < 8; n++)
    if (MP[e + off[n]] == 0.0) a = 0;
  double coefg = 0.0;
  if (a == 1) {
    double tmp = 0.0;
    for (int n = 0; n < 8; n++) tmp += MP[e + off[n]] * Ng[n];
    coefg = tmp;
  }
  return coefg;
}

/* K_G_d_g: degraded modulus g(d_g) * MP_g with d_g clamped to [0,1]. */
static double kgdg(const double* d, const double* MP, long e, const long off[8], const double* Ng,
                   double small_k) {
  double MP_g = gpmp(MP, e, off, Ng);
  double d_g = gpmp(d, e, off, Ng);
  if (d_g < 0.)
    d_g = 0.;
  else if (d_g > 1.)
    d_g = 1.;
  double g_d = (1. - small_k) * (1 - d_g) * (1 - d_g) + small_k;
  return g_d * MP_g;
}

/* MP_all_GAUSS_Point (mechanical_pcg.cpp:26-61). */
static void mat_gp(const shp* s, int finest, const short* choice, const double* bulK, const double* G,
                   const double* d, const double* Ke, const double* Ge, long e, const long off[8],
                   double small_k, double Kd[8], double Gd[8]) {
  for (int g = 0; g < 8; g++) {
    if (finest) {
      double K_g = gpmp(bulK, e, off, s->N[g]);
      double G_g = gpmp(G, e, off, s->N[g]);
      Kd[g] = (choice[e] == 0) ? kgdg(d, bulK, e, off, s->N[g], small_k) : K_g;
      Gd[g] = (choice[e] == 2) ? G_g : kgdg(d, G, e, off, s->N[g], small_k);
    } else {
      Kd[g] = Ke[e];
      Gd[g] = Ge[e];
    }
  }
}

/* epsilon_routine (mechanical_strain.cpp:15-35); u is a 3N block vector. */
static void strain_gp(const shp* s, const double* u, long N, long e, const long off[8], int g,
                      double eps[3][3]) {
  for (int c = 0; c < 3; c++)
    for (int m = 0; m < 3; m++) {
      double t = 0.0;
      for (int tf = 0; tf < 8; tf++) {
        double dc = u[c * N + e + off[tf]];
        double dm = u[m * N + e + off[tf]];
        t += 0.5 * (s->DN[c][g][tf] * dm + s->DN[m][g][tf] * dc);
      }
      eps[c][m] = t;
    }
}

static double trace3(double eps[3][3]) { return eps[0][0] + eps[1][1] + eps[2][2]; }

/* epsilon_dev (mechanical_strain.cpp:47-61). */
static double eps_dev(double eps[3][3]) {
  double ddp = 0.0;
  double third = (1.0 / 3.0) * trace3(eps);
  for (int c = 0; c < 3; c++)
    for (int m = 0; m < 3; m++) {
      if (c == m)
        ddp += (eps[c][m] - third) * (eps[c][m] - third);
      else
        ddp += eps[c][m] * eps[c][m];
    }
  return ddp;
}

/* Sigma_g (mechanical_stress.cpp:14-27). */
static void stress_gp(double sig[3][3], double eps[3][3], double K, double G, double tr) {
  for (int c = 0; c < 3; c++)
    for (int m = 0; m < 3; m++) {
      if (c == m)
        sig[c][m] = K * tr + 2.0 * G * (eps[c][m] - 1.0 / 3.0 * tr);
      else
        sig[c][m] = 2.0 * G * eps[c][m];
    }
}

/* Phi_positive / Phi_negative (strain_history.cpp:134-159). */
static double phi_pos(double K, double G, double eps[3][3]) {
  double tr = trace3(eps);
  double ddp = eps_dev(eps);
  if (tr >= 0) return 0.5 * K * tr * tr + G * ddp;
  return G * ddp;
}
static double phi_neg(double K, double eps[3][3]) {
  double tr = trace3(eps);
  if (tr >= 0) return 0.0;
  return 0.5 * K * tr * tr;
}

/* ------------------------------------------------------------------------- */
/* operators                                                                 */
/* ------------------------------------------------------------------------- */

/* Internal_Force[_element] (mechanical_pcg.cpp:114-191): Fi = K(d) u.  Element layers of one
 * parity touch disjoint node planes, so each parity runs in parallel without a critical section. */
int orc_internal_force(const orc_lvl* L, int finest, const double* u, const short* choice,
                       const double* bulK, const double* G, const double* d, const double* Ke,
                       const double* Ge, double small_k, double* Fi) {
  shp s;
  shape_init(&s, L->hx, L->hy, L->hz);
  long N = lvl_n(L), off[8];
  node_offsets(L, off);
  memset(Fi, 0, sizeof(double) * 3 * N);
  for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static)
    for (int k = color; k <= L->nz - 2; k += 2)
      for (int j = 0; j <= L->ny - 2; j++)
        for (int i = 0; i <= L->nx - 2; i++) {
          long e = i + (long)j * L->nx + (long)k * L->nx * L->ny;
          double Kd[8], Gd[8], sig[8][3][3], eps[3][3];
          mat_gp(&s, finest, choice, bulK, G, d, Ke, Ge, e, off, small_k, Kd, Gd);
          for (int g = 0; g < 8; g++) {
            strain_gp(&s, u, N, e, off, g, eps);
            double tr = trace3(eps);
            stress_gp(sig[g], eps, Kd[g], Gd[g], tr);
          }
          for (int sf = 0; sf < 8; sf++) {
            double fu = 0.0, fv = 0.0, fw = 0.0;
            for (int g = 0; g < 8; g++) {
              fu += s.wg * (sig[g][0][0] * s.DN[0][g][sf] + sig[g][1][0] * s.DN[1][g][sf] +
                            sig[g][2][0] * s.DN[2][g][sf]);
              fv += s.wg * (sig[g][0][1] * s.DN[0][g][sf] + sig[g][1][1] * s.DN[1][g][sf] +
                            sig[g][2][1] * s.DN[2][g][sf]);
              fw += s.wg * (sig[g][0][2] * s.DN[0][g][sf] + sig[g][1][2] * s.DN[1][g][sf] +
                            sig[g][2][2] * s.DN[2][g][sf]);
            }
            Fi[e + off[sf]] += fu;
            Fi[N + e + off[sf]] += fv;
            Fi[2 * N + e + off[sf]] += fw;
          }
        }
  }
  return 0;
}

/* PreM_u[_element] (mechanical_pcg.cpp:63-112): diagonal of K(d). */
int orc_prem_u(const orc_lvl* L, int finest, const short* choice, const double* bulK, const double* G,
               const double* d, const double* Ke, const double* Ge, double small_k, double* preM) {
  shp s;
  shape_init(&s, L->hx, L->hy, L->hz);
  long N = lvl_n(L), off[8];
  node_offsets(L, off);
  memset(preM, 0, sizeof(double) * 3 * N);
  for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static)
    for (int k = color; k <= L->nz - 2; k += 2)
      for (int j = 0; j <= L->ny - 2; j++)
        for (int i = 0; i <= L->nx - 2; i++) {
          long e = i + (long)j * L->nx + (long)k * L->nx * L->ny;
          double Kd[8], Gd[8];
          mat_gp(&s, finest, choice, bulK, G, d, Ke, Ge, e, off, small_k, Kd, Gd);
          for (int sf = 0; sf < 8; sf++) {
            double su = 0.0, sv = 0.0, sw = 0.0;
            for (int g = 0; g < 8; g++) {
              double d0 = s.DN[0][g][sf], d1 = s.DN[1][g][sf], d2 = s.DN[2][g][sf];
              su += s.wg * ((Kd[g] - 2. / 3. * Gd[g]) * d0 * d0 + 2. * Gd[g] * d0 * d0 +
                            Gd[g] * (d1 * d1 + d2 * d2));
              sv += s.wg * ((Kd[g] - 2. / 3. * Gd[g]) * d1 * d1 + 2. * Gd[g] * d1 * d1 +
                            Gd[g] * (d0 * d0 + d2 * d2));
              sw += s.wg * ((Kd[g] - 2. / 3. * Gd[g]) * d2 * d2 + 2. * Gd[g] * d2 * d2 +
                            Gd[g] * (d0 * d0 + d1 * d1));
            }
            preM[e + off[sf]] += su;
            preM[N + e + off[sf]] += sv;
            preM[2 * N + e + off[sf]] += sw;
          }
        }
  }
  return 0;
}

/* Fld[_element] (phase_field_pcg.cpp:61-103): Fi = A_d x,
 * A_d = sum_e wg [(2 H_e + gc_g/lc) N^T N + gc_g lc dN^T dN]. */
void orc_fld(const orc_lvl* L, const double* x, const double* H, const double* gc, double lc, double* Fi) {
  shp s;
  shape_init(&s, L->hx, L->hy, L->hz);
  long N = lvl_n(L), off[8];
  node_offsets(L, off);
  memset(Fi, 0, sizeof(double) * N);
  for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static)
    for (int k = color; k <= L->nz - 2; k += 2)
      for (int j = 0; j <= L->ny - 2; j++)
        for (int i = 0; i <= L->nx - 2; i++) {
          long e = i + (long)j * L->nx + (long)k * L->nx * L->ny;
          for (int sf = 0; sf < 8; sf++) {
            double acc = 0.0;
            for (int g = 0; g < 8; g++) {
              double gc_g = gpmp(gc, e, off, s.N[g]);
              for (int tf = 0; tf < 8; tf++)
                acc += s.wg *
                       ((2.0 * H[e] + gc_g / lc) * s.N[g][sf] * s.N[g][tf] +
                        gc_g * lc *
                            (s.DN[0][g][sf] * s.DN[0][g][tf] + s.DN[1][g][sf] * s.DN[1][g][tf] +
                             s.DN[2][g][sf] * s.DN[2][g][tf])) *
                       x[e + off[tf]];
            }
            Fi[e + off[sf]] += acc;
          }
        }
  }
}

/* Md_element / Precondition_M (phase_field_pcg.cpp:20-59): diagonal of A_d. */
void orc_precondition_m(const orc_lvl* L, const double* H, const double* gc, double lc, double* Md) {
  shp s;
  shape_init(&s, L->hx, L->hy, L->hz);
  long N = lvl_n(L), off[8];
  node_offsets(L, off);
  memset(Md, 0, sizeof(double) * N);
  for (int color = 0; color < 2; ++color) {
#pragma omp parallel for schedule(static)
    for (int k = color; k <= L->nz - 2; k += 2)
      for (int j = 0; j <= L->ny - 2; j++)
        for (int i = 0; i <= L->nx - 2; i++) {
          long e = i + (long)j * L->nx + (long)k * L->nx * L->ny;
          for (int sf = 0; sf < 8; sf++) {
            double acc = 0.0;
            for (int g = 0; g < 8; g++) {
              double gc_g = gpmp(gc, e, off, s.N[g]);
              acc += s.wg * ((2. * H[e] + gc_g / lc) * s.N[g][sf] * s.N[g][sf] +
                             gc_g * lc *
                                 (s.DN[0][g][sf] * s.DN[0][g][sf] + s.DN[1][g][sf] * s.DN[1][g][sf] +
                                  s.DN[2][g][sf] * s.DN[2][g][sf]));
            }
            Md[e + off[sf]] += acc;
          }
        }
  }
}

/* ------------------------------------------------------------------------- */
/* inter-grid transfers (multigrid_intergrid.cpp)                            */
/* ------------------------------------------------------------------------- */

/* solution_injection (:25-90): uc(i,j,k) = uf(2i,2j,2k). */
void orc_injection(const orc_lvl* Lc, const orc_lvl* Lf, const double* uf, double* uc) {
#pragma omp parallel for schedule(static)
  for (int kc = 0; kc < Lc->nz; kc++)
    for (int jc = 0; jc < Lc->ny; jc++)
      for (int ic = 0; ic < Lc->nx; ic++)
        uc[ic + (long)jc * Lc->nx + (long)kc * Lc->nx * Lc->ny] =
            uf[2 * ic + (long)(2 * jc) * Lf->nx + (long)(2 * kc) * Lf->nx * Lf->ny];
}

/* coarsen_f_standard_routine (:124-342): fc = Fic + full weighting of rf (27 points, weights
 * 1/8 x {1,2,4,8}), neighbours outside the fine grid count as 0. */
void orc_restrict(const orc_lvl* Lc, const orc_lvl* Lf, const double* rf, const double* Fic, double* fc) {
  int Xl = Lf->nx - 2, Yl = Lf->ny - 2, Zl = Lf->nz - 2;
  long sy = Lf->nx, sz = (long)Lf->nx * Lf->ny;
#define RF(a, b, c) rf[(a) + (long)(b) * sy + (long)(c) * sz]
#pragma omp parallel for schedule(static)
  for (int ic = 0; ic < Lc->nx; ic++)
    for (int jc = 0; jc < Lc->ny; jc++)
      for (int kc = 0; kc < Lc->nz; kc++) {
        int x = 2 * ic, y = 2 * jc, z = 2 * kc;
        double r11 = (x < 1 || y < 1 || z < 1) ? 0.0 : RF(x - 1, y - 1, z - 1);
        double r12 = (x < 1 || y < 1 || z > Zl) ? 0.0 : RF(x - 1, y - 1, z + 1);
        double r13 = (x < 1 || y > Yl || z < 1) ? 0.0 : RF(x - 1, y + 1, z - 1);
        double r14 = (x < 1 || y > Yl || z > Zl) ? 0.0 : RF(x - 1, y + 1, z + 1);
        double r15 = (x > Xl || y < 1 || z < 1) ? 0.0 : RF(x + 1, y - 1, z - 1);
        double r16 = (x > Xl || y < 1 || z > Zl) ? 0.0 : RF(x + 1, y - 1, z + 1);
        double r17 = (x > Xl || y > Yl || z < 1) ? 0.0 : RF(x + 1, y + 1, z - 1);
        double r18 = (x > Xl || y > Yl || z > Zl) ? 0.0 : RF(x + 1, y + 1, z + 1);
        double r21 = (x < 1 || y < 1) ? 0.0 : RF(x - 1, y - 1, z);
        double r22 = (x < 1 || y > Yl) ? 0.0 : RF(x - 1, y + 1, z);
        double r23 = (x > Xl || y < 1) ? 0.0 : RF(x + 1, y - 1, z);
        double r24 = (x > Xl || y > Yl) ? 0.0 : RF(x + 1, y + 1, z);
        double r25 = (x < 1 || z < 1) ? 0.0 : RF(x - 1, y, z - 1);
        double r26 = (x < 1 || z > Zl) ? 0.0 : RF(x - 1, y, z + 1);
        double r27 = (x > Xl || z < 1) ? 0.0 : RF(x + 1, y, z - 1);
        double r28 = (x > Xl || z > Zl) ? 0.0 : RF(x + 1, y, z + 1);
        double r29 = (y < 1 || z < 1) ? 0.0 : RF(x, y - 1, z - 1);
        double r210 = (y < 1 || z > Zl) ? 0.0 : RF(x, y - 1, z + 1);
        double r211 = (y > Yl || z < 1) ? 0.0 : RF(x, y + 1, z - 1);
        double r212 = (y > Yl || z > Zl) ? 0.0 : RF(x, y + 1, z + 1);
        double r41 = (z < 1) ? 0.0 : RF(x, y, z - 1);
        double r42 = (z > Zl) ? 0.0 : RF(x, y, z + 1);
        double r43 = (y < 1) ? 0.0 : RF(x, y - 1, z);
        double r44 = (y > Yl) ? 0.0 : RF(x, y + 1, z);
        double r45 = (x < 1) ? 0.0 : RF(x - 1, y, z);
        double r46 = (x > Xl) ? 0.0 : RF(x + 1, y, z);
        double r8 = RF(x, y, z);
        long ci = ic + (long)jc * Lc->nx + (long)kc * Lc->nx * Lc->ny;
        fc[ci] = Fic[ci] + 0.125 * (r11 + r12 + r13 + r14 + r15 + r16 + r17 + r18 +
                                    2.0 * (r21 + r22 + r23 + r24 + r25 + r26 + r27 + r28 + r29 + r210 +
                                           r211 + r212) +
                                    4.0 * (r41 + r42 + r43 + r44 + r45 + r46) + 8.0 * r8);
      }
#undef RF
}

/* refine_standard_routine (:416-520): uf += trilinear prolongation of (uc - ucold). */
void orc_prolong(const orc_lvl* Lc, const orc_lvl* Lf, const double* uc, const double* ucold, double* uf) {
  long csy = Lc->nx, csz = (long)Lc->nx * Lc->ny;
  long fsy = Lf->nx, fsz = (long)Lf->nx * Lf->ny;
#define E(a, b, c) (uc[(a) + (long)(b) * csy + (long)(c) * csz] - ucold[(a) + (long)(b) * csy + (long)(c) * csz])
#define UF(a, b, c) uf[(a) + (long)(b) * fsy + (long)(c) * fsz]
#pragma omp parallel for schedule(static)
  for (int ic = 0; ic < Lc->nx; ic++)
    for (int jc = 0; jc < Lc->ny; jc++)
      for (int kc = 0; kc < Lc->nz; kc++) {
        int x = 2 * ic, y = 2 * jc, z = 2 * kc;
        UF(x, y, z) += E(ic, jc, kc);
        if (x > 0) UF(x - 1, y, z) += 0.5 * (E(ic, jc, kc) + E(ic - 1, jc, kc));
        if (y > 0) UF(x, y - 1, z) += 0.5 * (E(ic, jc, kc) + E(ic, jc - 1, kc));
        if (z > 0) UF(x, y, z - 1) += 0.5 * (E(ic, jc, kc) + E(ic, jc, kc - 1));
        if (x > 0 && y > 0)
          UF(x - 1, y - 1, z) +=
              0.25 * (E(ic, jc, kc) + E(ic, jc - 1, kc) + E(ic - 1, jc, kc) + E(ic - 1, jc - 1, kc));
        if (x > 0 && z > 0)
          UF(x - 1, y, z - 1) +=
              0.25 * (E(ic, jc, kc) + E(ic - 1, jc, kc - 1) + E(ic, jc, kc - 1) + E(ic - 1, jc, kc));
        if (y > 0 && z > 0)
          UF(x, y - 1, z - 1) +=
              0.25 * (E(ic, jc, kc) + E(ic, jc - 1, kc - 1) + E(ic, jc, kc - 1) + E(ic, jc - 1, kc));
        if (x > 0 && y > 0 && z > 0)
          UF(x - 1, y - 1, z - 1) +=
              0.125 * (E(ic, jc, kc) + E(ic, jc - 1, kc) + E(ic - 1, jc, kc) + E(ic - 1, jc - 1, kc) +
                       E(ic, jc, kc - 1) + E(ic - 1, jc, kc - 1) + E(ic, jc - 1, kc - 1) +
                       E(ic - 1, jc - 1, kc - 1));
      }
#undef E
#undef UF
}

/* ------------------------------------------------------------------------- */
/* hierarchy state                                                           */
/* ------------------------------------------------------------------------- */

struct orc_state {
  orc_geom geo;
  double *bulK[ORC_MAXL], *G[ORC_MAXL], *gc[ORC_MAXL], *d[ORC_MAXL], *H[ORC_MAXL], *fd[ORC_MAXL];
  double *Ke[ORC_MAXL], *Ge[ORC_MAXL], *R[ORC_MAXL], *dold[ORC_MAXL];
  double *u[ORC_MAXL], *fu[ORC_MAXL], *ru[ORC_MAXL], *uold[ORC_MAXL];
  short* choice[ORC_MAXL];
  double* d_old;
  double f_norm, fd_norm, Ue, Ut, dU, uprop;
  int choice_quirk;
};

orc_state* orc_state_create(int maxlevel, const int* enb, const double* x0, const int* roi) {
  if (maxlevel < 0 || maxlevel >= ORC_MAXL) return NULL;
  orc_state* s = (orc_state*)calloc(1, sizeof *s);
  orc_geom_init(&s->geo, maxlevel, enb, x0, roi);
  for (int l = 0; l <= maxlevel; ++l) {
    long N = lvl_n(&s->geo.lv[l]);
    s->bulK[l] = calloc(N, 8); s->G[l] = calloc(N, 8); s->gc[l] = calloc(N, 8);
    s->d[l] = calloc(N, 8); s->H[l] = calloc(N, 8); s->fd[l] = calloc(N, 8);
    s->Ke[l] = calloc(N, 8); s->Ge[l] = calloc(N, 8); s->R[l] = calloc(N, 8);
    s->dold[l] = calloc(N, 8);
    s->u[l] = calloc(3 * N, 8); s->fu[l] = calloc(3 * N, 8); s->ru[l] = calloc(3 * N, 8);
    s->uold[l] = calloc(3 * N, 8);
    s->choice[l] = calloc(N, sizeof(short));
  }
  s->d_old = calloc(lvl_n(&s->geo.lv[maxlevel]), 8);
  s->choice_quirk = 1;
  return s;
}

void orc_state_destroy(orc_state* s) {
  if (!s) return;
  for (int l = 0; l <= s->geo.maxlevel; ++l) {
    free(s->bulK[l]); free(s->G[l]); free(s->gc[l]); free(s->d[l]); free(s->H[l]); free(s->fd[l]);
    free(s->Ke[l]); free(s->Ge[l]); free(s->R[l]); free(s->dold[l]);
    free(s->u[l]); free(s->fu[l]); free(s->ru[l]); free(s->uold[l]); free(s->choice[l]);
  }
  free(s->d_old);
  free(s);
}

const orc_geom* orc_state_geom(const orc_state* s) { return &s->geo; }
void orc_set_choice_quirk(orc_state* s, int reproduce) { s->choice_quirk = reproduce != 0; }

static double** scalar_of(orc_state* s, int f) {
  switch (f) {
    case ORC_BULK: return s->bulK;
    case ORC_G: return s->G;
    case ORC_GC: return s->gc;
    case ORC_D: return s->d;
    case ORC_H: return s->H;
    case ORC_FD: return s->fd;
    case ORC_KE: return s->Ke;
    case ORC_GE: return s->Ge;
    case ORC_R: return s->R;
    case ORC_DOLD: return s->dold;
    default: return NULL;
  }
}
static double** vector_of(orc_state* s, int f) {
  switch (f) {
    case ORC_U: return s->u;
    case ORC_FU: return s->fu;
    case ORC_RU: return s->ru;
    case ORC_UOLD: return s->uold;
    default: return NULL;
  }
}
static double* array_of(orc_state* s, int f, int l, int comp) {
  if (l < 0 || l > s->geo.maxlevel) return NULL;
  long N = lvl_n(&s->geo.lv[l]);
  if (f == ORC_DOLDF) return l == s->geo.maxlevel ? s->d_old : NULL;
  double** a = scalar_of(s, f);
  if (a) return a[l];
  a = vector_of(s, f);
  if (a && comp >= 0 && comp < 3) return a[l] + comp * N;
  return NULL;
}

int orc_set(orc_state* s, int field, int level, int comp, const double* src) {
  double* a = array_of(s, field, level, comp);
  if (!a) return -1;
  memcpy(a, src, sizeof(double) * lvl_n(&s->geo.lv[level]));
  return 0;
}
int orc_get(orc_state* s, int field, int level, int comp, double* dst) {
  double* a = array_of(s, field, level, comp);
  if (!a) return -1;
  memcpy(dst, a, sizeof(double) * lvl_n(&s->geo.lv[level]));
  return 0;
}
int orc_set_choice(orc_state* s, int level, const short* src) {
  memcpy(s->choice[level], src, sizeof(short) * lvl_n(&s->geo.lv[level]));
  return 0;
}
int orc_get_choice(orc_state* s, int level, short* dst) {
  memcpy(dst, s->choice[level], sizeof(short) * lvl_n(&s->geo.lv[level]));
  return 0;
}
void orc_state_scalars(orc_state* s, double* s6) {
  s6[0] = s->f_norm; s6[1] = s->fd_norm; s6[2] = s->Ue; s6[3] = s->Ut; s6[4] = s->dU; s6[5] = s->uprop;
}
void orc_set_state_scalars(orc_state* s, const double* s6) {
  s->f_norm = s6[0]; s->fd_norm = s6[1]; s->Ue = s6[2]; s->Ut = s6[3]; s->dU = s6[4]; s->uprop = s6[5];
}

/* grid_norm / vv_product (pcg_utilities.cpp:16-58): squared norm and dot over the whole level. */
static double dot_n(const double* a, const double* b, long n) {
  double ss = 0.0;
  for (long i = 0; i < n; ++i) ss += a[i] * b[i];
  return ss;
}

int orc_st_internal_force(orc_state* s, int l, int src, int dst, double small_k) {
  double** a = vector_of(s, src);
  double** o = vector_of(s, dst);
  if (!a || !o || a == o) return -1;
  return orc_internal_force(&s->geo.lv[l], l == s->geo.maxlevel, a[l], s->choice[l], s->bulK[l], s->G[l],
                            s->d[l], s->Ke[l], s->Ge[l], small_k, o[l]);
}
int orc_st_prem_u(orc_state* s, int l, int dst, double small_k) {
  double** o = vector_of(s, dst);
  if (!o) return -1;
  return orc_prem_u(&s->geo.lv[l], l == s->geo.maxlevel, s->choice[l], s->bulK[l], s->G[l], s->d[l],
                    s->Ke[l], s->Ge[l], small_k, o[l]);
}
int orc_st_fld(orc_state* s, int l, int src, int dst, double lc) {
  double** a = scalar_of(s, src);
  double** o = scalar_of(s, dst);
  if (!a || !o || a == o) return -1;
  orc_fld(&s->geo.lv[l], a[l], s->H[l], s->gc[l], lc, o[l]);
  return 0;
}
int orc_st_precondition_m(orc_state* s, int l, int dst, double lc) {
  double** o = scalar_of(s, dst);
  if (!o) return -1;
  orc_precondition_m(&s->geo.lv[l], s->H[l], s->gc[l], lc, o[l]);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* boundary conditions (boundary_conditions.cpp:14-154)                      */
/* ------------------------------------------------------------------------- */

/* Dirichlet node sets are selected by floating-point coordinate equality; coordinates are
 * get_coordinate (:14-18) for one rank: origin + index*h.  kind: 0 = set u (Dirichlet_BD),
 * 1 = copy Fi into f (Dirichlet_force_u), 2 = zero r (Dirichlet_residual_u). */
static void bc_apply(orc_state* s, int l, double* v, const double* fi, int kind, double Ut) {
  const orc_lvl* L = &s->geo.lv[l];
  const double* B = s->geo.box;
  long N = lvl_n(L);
  for (int k = 0; k <= L->nz - 1; k++) {
    double z = B[4] + k * L->hz;
    for (int j = 0; j <= L->ny - 1; j++) {
      double y = B[2] + j * L->hy;
      for (int i = 0; i <= L->nx - 1; i++) {
        double x = B[0] + i * L->hx;
        long n = i + (long)j * L->nx + (long)k * L->nx * L->ny;
        if (z == B[4] && x == 0.5 * (B[0] + B[1]) && y == B[2])
          v[n] = kind == 1 ? fi[n] : 0.0;
        if (z == B[4] && x == B[1] && y == 0.5 * (B[2] + B[3]))
          v[N + n] = kind == 1 ? fi[N + n] : 0.0;
        if (z == B[4]) v[2 * N + n] = kind == 1 ? fi[2 * N + n] : 0.0;
        if (z == B[5]) v[2 * N + n] = kind == 1 ? fi[2 * N + n] : (kind == 0 ? Ut : 0.0);
      }
    }
  }
}

int orc_dirichlet_bd(orc_state* s, int l, int field, double Ut) {
  double** v = vector_of(s, field);
  if (!v) return -1;
  bc_apply(s, l, v[l], NULL, 0, Ut);
  return 0;
}
int orc_dirichlet_force(orc_state* s, int l, int f_field, int fi_field) {
  double** f = vector_of(s, f_field);
  double** fi = vector_of(s, fi_field);
  if (!f || !fi) return -1;
  bc_apply(s, l, f[l], fi[l], 1, 0.0);
  return 0;
}
int orc_dirichlet_residual(orc_state* s, int l, int field) {
  double** v = vector_of(s, field);
  if (!v) return -1;
  bc_apply(s, l, v[l], NULL, 2, 0.0);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* smoothers                                                                 */
/* ------------------------------------------------------------------------- */

/* Initial_residual_u (mechanical_pcg.cpp:193-220). */
double orc_initial_residual_u(orc_state* s, int l, double small_k) {
  const orc_lvl* L = &s->geo.lv[l];
  long N = lvl_n(L);
  double* Fi = malloc(sizeof(double) * 3 * N);
  orc_internal_force(L, l == s->geo.maxlevel, s->u[l], s->choice[l], s->bulK[l], s->G[l], s->d[l], s->Ke[l],
                     s->Ge[l], small_k, Fi);
  for (long i = 0; i < 3 * N; ++i) s->ru[l][i] = s->fu[l][i] - Fi[i];
  bc_apply(s, l, s->ru[l], NULL, 2, 0.0);
  double r = 0.0;
  for (int di = 0; di < 3; ++di) r += dot_n(s->ru[l] + di * N, s->ru[l] + di * N, N);
  free(Fi);
  return r;
}

/* pcg_u (mechanical_pcg.cpp:223-330): restarted Jacobi-preconditioned CG, NB_relax iterations.
 * Returns the iterations run, or -1 where the reference throws (zero diagonal entry). */
int orc_pcg_u(orc_state* s, int l, double small_k, double Ut, int nb_relax, int t, double* f_norm) {
  const orc_lvl* L = &s->geo.lv[l];
  long N = lvl_n(L);
  int finest = l == s->geo.maxlevel;
  double* preM = calloc(3 * N, 8);
  double* Fi = calloc(3 * N, 8);
  double* z = calloc(3 * N, 8);
  double* p = calloc(3 * N, 8);
  double* u = s->u[l];
  double* ru = s->ru[l];
  double* fu = s->fu[l];
  int rc = nb_relax;
  bc_apply(s, l, u, NULL, 0, Ut);
  orc_internal_force(L, finest, u, s->choice[l], s->bulK[l], s->G[l], s->d[l], s->Ke[l], s->Ge[l], small_k, Fi);
  if (t == 0 && finest) {
    bc_apply(s, l, fu, Fi, 1, 0.0);
    *f_norm = 0.0;
    for (int di = 0; di < 3; ++di) *f_norm += dot_n(fu + di * N, fu + di * N, N);
  }
  for (long i = 0; i < 3 * N; ++i) ru[i] = fu[i] - Fi[i];
  bc_apply(s, l, ru, NULL, 2, 0.0);
  orc_prem_u(L, finest, s->choice[l], s->bulK[l], s->G[l], s->d[l], s->Ke[l], s->Ge[l], small_k, preM);
  double rz_old = 0.0;
  for (int it = 0; it < nb_relax; it++) {
    for (long i = 0; i < 3 * N; ++i) {
      if (preM[i] == 0.0) { rc = -1; goto done; }
      z[i] = ru[i] / preM[i];
    }
    double rz_new = 0.0;
    for (int di = 0; di < 3; ++di) rz_new += dot_n(ru + di * N, z + di * N, N);
    double beta = (it == 0) ? 0.0 : rz_new / rz_old;
    for (long i = 0; i < 3 * N; ++i) p[i] = z[i] + p[i] * beta;
    orc_internal_force(L, finest, p, s->choice[l], s->bulK[l], s->G[l], s->d[l], s->Ke[l], s->Ge[l], small_k, Fi);
    double pw = 0.0;
    for (int di = 0; di < 3; ++di) pw += dot_n(p + di * N, Fi + di * N, N);
    double alpha = rz_new / pw;
    for (long i = 0; i < 3 * N; ++i) {
      u[i] = u[i] + p[i] * alpha;
      ru[i] = ru[i] - Fi[i] * alpha;
    }
    bc_apply(s, l, ru, NULL, 2, 0.0);
    rz_old = rz_new;
  }
done:
  free(preM); free(Fi); free(z); free(p);
  return rc;
}

/* initial_residual (phase_field_pcg.cpp:106-131). */
double orc_initial_residual_d(orc_state* s, int l, double lc) {
  const orc_lvl* L = &s->geo.lv[l];
  long N = lvl_n(L);
  double* Fi = malloc(sizeof(double) * N);
  orc_fld(L, s->d[l], s->H[l], s->gc[l], lc, Fi);
  for (long i = 0; i < N; ++i) s->R[l][i] = s->fd[l][i] - Fi[i];
  double r = dot_n(s->R[l], s->R[l], N);
  free(Fi);
  return r;
}

/* pcg_d (phase_field_pcg.cpp:133-214).  fd_norm is rewritten on every call (:163). */
int orc_pcg_d(orc_state* s, int l, double lc, int nb_relax, int t, double* fd_norm) {
  (void)t;
  const orc_lvl* L = &s->geo.lv[l];
  long N = lvl_n(L);
  double* preM = calloc(N, 8);
  double* Fi = calloc(N, 8);
  double* z = calloc(N, 8);
  double* p = calloc(N, 8);
  double* d = s->d[l];
  double* R = s->R[l];
  double* fd = s->fd[l];
  int rc = nb_relax;
  orc_precondition_m(L, s->H[l], s->gc[l], lc, preM);
  orc_fld(L, d, s->H[l], s->gc[l], lc, Fi);
  *fd_norm = dot_n(fd, fd, N);
  for (long i = 0; i < N; ++i) R[i] = fd[i] - Fi[i];
  double rz_old = 0.0;
  for (int it = 0; it < nb_relax; it++) {
    for (long i = 0; i < N; ++i) {
      if (preM[i] == 0.0) { rc = -1; goto done; }
      z[i] = R[i] / preM[i];
    }
    double rz_new = dot_n(R, z, N);
    double beta = (it == 0) ? 0.0 : rz_new / rz_old;
    for (long i = 0; i < N; ++i) p[i] = z[i] + p[i] * beta;
    orc_fld(L, p, s->H[l], s->gc[l], lc, Fi);
    double pw = dot_n(p, Fi, N);
    double alpha = rz_new / pw;
    for (long i = 0; i < N; ++i) {
      d[i] = d[i] + p[i] * alpha;
      R[i] = R[i] - Fi[i] * alpha;
    }
    rz_old = rz_new;
  }
done:
  free(preM); free(Fi); free(z); free(p);
  return rc;
}

/* ------------------------------------------------------------------------- */
/* V-cycles (mechanical_multigrid.cpp:18-54, phase_field_multigrid.cpp:18-44) */
/* ------------------------------------------------------------------------- */

/* Returns the smoother iterations run on all levels, or -1. */
int orc_cycle_u(orc_state* s, int l, const int* mg5, double small_k, double Ut, int t, double* f_norm) {
  int nu0 = mg5[0], nu1 = mg5[1], nu2 = mg5[2], gamma = mg5[3];
  if (l == 0) return orc_pcg_u(s, 0, small_k, Ut, nu0, t, f_norm);
  int it = 0, r;
  if ((r = orc_pcg_u(s, l, small_k, Ut, nu1, t, f_norm)) < 0) return -1;
  it += r;
  const orc_lvl* Lc = &s->geo.lv[l - 1];
  const orc_lvl* Lf = &s->geo.lv[l];
  long Nc = lvl_n(Lc), Nf = lvl_n(Lf);
  /* coarsen_u (multigrid_intergrid.cpp:106-121) */
  for (int di = 0; di < 3; ++di) orc_injection(Lc, Lf, s->u[l] + di * Nf, s->u[l - 1] + di * Nc);
  bc_apply(s, l - 1, s->u[l - 1], NULL, 0, Ut);
  memcpy(s->uold[l - 1], s->u[l - 1], sizeof(double) * 3 * Nc);
  /* coarsen_fu (:374-413) */
  double* Fic = malloc(sizeof(double) * 3 * Nc);
  orc_internal_force(Lc, 0, s->u[l - 1], s->choice[l - 1], s->bulK[l - 1], s->G[l - 1], s->d[l - 1],
                     s->Ke[l - 1], s->Ge[l - 1], small_k, Fic);
  for (int di = 0; di < 3; ++di)
    orc_restrict(Lc, Lf, s->ru[l] + di * Nf, Fic + di * Nc, s->fu[l - 1] + di * Nc);
  free(Fic);
  for (int j = 1; j <= gamma; j++) {
    if ((r = orc_cycle_u(s, l - 1, mg5, small_k, Ut, t, f_norm)) < 0) return -1;
    it += r;
  }
  /* refine_u (:536-549) */
  for (int di = 0; di < 3; ++di)
    orc_prolong(Lc, Lf, s->u[l - 1] + di * Nc, s->uold[l - 1] + di * Nc, s->u[l] + di * Nf);
  bc_apply(s, l, s->u[l], NULL, 0, Ut);
  if ((r = orc_pcg_u(s, l, small_k, Ut, nu2, t, f_norm)) < 0) return -1;
  return it + r;
}

int orc_cycle_d(orc_state* s, int l, const int* mg5, double lc, int t, double* fd_norm) {
  int nu0 = mg5[0], nu1 = mg5[1], nu2 = mg5[2], gamma = mg5[3];
  if (l == 0) return orc_pcg_d(s, 0, lc, nu0, t, fd_norm);
  int it = 0, r;
  if ((r = orc_pcg_d(s, l, lc, nu1, t, fd_norm)) < 0) return -1;
  it += r;
  const orc_lvl* Lc = &s->geo.lv[l - 1];
  const orc_lvl* Lf = &s->geo.lv[l];
  long Nc = lvl_n(Lc);
  /* coarsen_d (multigrid_intergrid.cpp:92-103) */
  orc_injection(Lc, Lf, s->d[l], s->d[l - 1]);
  memcpy(s->dold[l - 1], s->d[l - 1], sizeof(double) * Nc);
  /* coarsen_f_d (:345-371) */
  double* Fic = malloc(sizeof(double) * Nc);
  orc_fld(Lc, s->d[l - 1], s->H[l - 1], s->gc[l - 1], lc, Fic);
  orc_restrict(Lc, Lf, s->R[l], Fic, s->fd[l - 1]);
  free(Fic);
  for (int j = 1; j <= gamma; j++) {
    if ((r = orc_cycle_d(s, l - 1, mg5, lc, t, fd_norm)) < 0) return -1;
    it += r;
  }
  /* refine_d (:523-533) */
  orc_prolong(Lc, Lf, s->d[l - 1], s->dold[l - 1], s->d[l]);
  /* post-smoothing runs nu2 calls of nu2 iterations (phase_field_multigrid.cpp:41-42) */
  for (int i = 1; i <= nu2; i++) {
    if ((r = orc_pcg_d(s, l, lc, nu2, t, fd_norm)) < 0) return -1;
    it += r;
  }
  return it;
}

/* ------------------------------------------------------------------------- */
/* material selection and coarse element material                            */
/* ------------------------------------------------------------------------- */

/* MP_choice_element (material_selection.cpp:19-45) at the element whose first node is flat index e. */
static short choice_elem(const shp* s, const double* u, long N, const double* bulK, const double* G, long e,
                         const long off[8]) {
  double tr = 0.0, pp = 0.0, pn = 0.0, eps[3][3];
  for (int g = 0; g < 8; g++) {
    double K_g = gpmp(bulK, e, off, s->N[g]);
    double G_g = gpmp(G, e, off, s->N[g]);
    strain_gp(s, u, N, e, off, g, eps);
    tr += trace3(eps);
    pp += phi_pos(K_g, G_g, eps);
    pn += phi_neg(K_g, eps);
  }
  short c = 0;
  if (tr >= 0.0) c = 0;
  if (tr < 0.0) c = 1;
  if (pp < pn) c = 2;
  return c;
}

/* Whether the reference's MP_choice loop (material_selection.cpp:59-63) writes flat slot b.
 * That loop passes an index bounded by the y extent as x (i <= ny-2) and one bounded by the x
 * extent as y (j <= nx-2); every access is a flat offset from b = i + j*nx + k*nx*ny, so the
 * slots written are exactly those b (possibly reached from a lower k), and each holds the value
 * computed at that flat base.  For nx == ny this is every element. */
static int choice_in_image(long b, long nx, long ny, long nz) {
  long P = nx * ny, z = b / P, rmax = (ny - 2) + (nx - 2) * nx;
  for (long kp = (z < nz - 2 ? z : nz - 2); kp >= 0; --kp) {
    long r = b - kp * P;
    if (r > rmax) break;
    long jlo = r - (ny - 2) <= 0 ? 0 : (r - (ny - 2) + nx - 1) / nx;
    long jhi = r / nx < nx - 2 ? r / nx : nx - 2;
    if (jlo <= jhi) return 1;
  }
  return 0;
}

/* MP_choice (material_selection.cpp:47-65) on every level of a freshly zeroed field.  Consumers read
 * element slots only (material_selection.cpp:80-87, mechanical_pcg.cpp:41-53); an element slot holds
 * its regime when the reference's loop reaches it (choice_in_image) and 0 otherwise.  Slots that are
 * not elements are left 0 (the reference may write values read across the array end there when
 * nx > ny).  choice_quirk = 0 computes every element. */
void orc_mp_choice(orc_state* s) {
  for (int l = s->geo.maxlevel; l >= 0; l--) {
    const orc_lvl* L = &s->geo.lv[l];
    shp sh;
    shape_init(&sh, L->hx, L->hy, L->hz);
    long N = lvl_n(L), off[8];
    node_offsets(L, off);
    memset(s->choice[l], 0, sizeof(short) * N);
    long nx = L->nx, ny = L->ny, nz = L->nz;
    int quirk = s->choice_quirk;
#pragma omp parallel for schedule(static)
    for (int k = 0; k <= L->nz - 2; k++)
      for (long j = 0; j <= ny - 2; j++)
        for (long i = 0; i <= nx - 2; i++) {
          long e = i + j * nx + (long)k * nx * ny;
          if (!quirk || choice_in_image(e, nx, ny, nz))
            s->choice[l][e] = choice_elem(&sh, s->u[l], N, s->bulK[l], s->G[l], e, off);
        }
  }
}

/* MP_element / MP_all_element (material_selection.cpp:67-116): finest element-mean degraded K, G. */
void orc_mp_all_element(orc_state* s, double small_k) {
  int l = s->geo.maxlevel;
  const orc_lvl* L = &s->geo.lv[l];
  shp sh;
  shape_init(&sh, L->hx, L->hy, L->hz);
  long off[8];
  node_offsets(L, off);
  const double *bulK = s->bulK[l], *G = s->G[l], *d = s->d[l];
  const short* ch = s->choice[l];
#pragma omp parallel for schedule(static)
  for (int k = 0; k <= L->nz - 2; k++)
    for (int j = 0; j <= L->ny - 2; j++)
      for (int i = 0; i <= L->nx - 2; i++) {
        long e = i + (long)j * L->nx + (long)k * L->nx * L->ny;
        double K_e = 0., G_e = 0.;
        for (int g = 0; g < 8; g++) {
          double K_g = gpmp(bulK, e, off, sh.N[g]);
          double G_g = gpmp(G, e, off, sh.N[g]);
          if (ch[e] == 0)
            K_e += kgdg(d, bulK, e, off, sh.N[g], small_k);
          else
            K_e += K_g;
          if (ch[e] == 2)
            G_e += G_g;
          else
            G_e += kgdg(d, G, e, off, sh.N[g], small_k);
        }
        s->Ke[l][e] = 0.125 * K_e;
        s->Ge[l][e] = 0.125 * G_e;
      }
}

/* coarse_voigt / coarse_reuss (material_coarse_element.cpp:20-82) on coarse element slots. */
static void coarse_vr_elem(const orc_lvl* Lc, const orc_lvl* Lf, const double* Hf, double* Hv, double* Hr) {
  long fsy = Lf->nx, fsz = (long)Lf->nx * Lf->ny;
#define HF(a, b, c) Hf[(a) + (long)(b) * fsy + (long)(c) * fsz]
#pragma omp parallel for schedule(static)
  for (int ic = 0; ic <= Lc->nx - 2; ic++)
    for (int jc = 0; jc <= Lc->ny - 2; jc++)
      for (int kc = 0; kc <= Lc->nz - 2; kc++) {
        int x = 2 * ic, y = 2 * jc, z = 2 * kc;
        long ci = ic + (long)jc * Lc->nx + (long)kc * Lc->nx * Lc->ny;
        if (Hv)
          Hv[ci] = 0.125 * (HF(x, y, z) + HF(x + 1, y, z) + HF(x, y + 1, z) + HF(x + 1, y + 1, z) +
                            HF(x, y, z + 1) + HF(x + 1, y, z + 1) + HF(x, y + 1, z + 1) +
                            HF(x + 1, y + 1, z + 1));
        if (Hr)
          Hr[ci] = 8. / (1. / HF(x, y, z) + 1. / HF(x + 1, y, z) + 1. / HF(x, y + 1, z) +
                         1. / HF(x + 1, y + 1, z) + 1. / HF(x, y, z + 1) + 1. / HF(x + 1, y, z + 1) +
                         1. / HF(x, y + 1, z + 1) + 1. / HF(x + 1, y + 1, z + 1));
      }
#undef HF
}

/* VR_all_level (material_coarse_element.cpp:86-102): Hill mean 0.5*(0.5*(V+R) + sqrt(V*R)). */
int orc_vr_all_level(orc_state* s, int field) {
  double** H = scalar_of(s, field);
  if (!H) return -1;
  for (int l = s->geo.maxlevel; l > 0; l--) {
    const orc_lvl* Lc = &s->geo.lv[l - 1];
    long Nc = lvl_n(Lc);
    double* Hv = calloc(Nc, 8);
    double* Hr = calloc(Nc, 8);
    coarse_vr_elem(Lc, &s->geo.lv[l], H[l], Hv, Hr);
    for (long i = 0; i < Nc; ++i) H[l - 1][i] = 0.5 * (0.5 * (Hv[i] + Hr[i]) + sqrt(Hv[i] * Hr[i]));
    free(Hv);
    free(Hr);
  }
  return 0;
}

/* Voigt_all_level (material_coarse_element.cpp:106-118). */
int orc_voigt_all_level(orc_state* s, int field) {
  double** H = scalar_of(s, field);
  if (!H) return -1;
  for (int l = s->geo.maxlevel; l > 0; l--) coarse_vr_elem(&s->geo.lv[l - 1], &s->geo.lv[l], H[l], H[l - 1], NULL);
  return 0;
}

/* voight / reuss / coarse_VR (image_input.cpp:144-260): nodal 27-point Hill mean to coarse levels,
 * neighbour indices clamped to the fine grid. */
int orc_coarse_vr(orc_state* s, int field) {
  double** M = scalar_of(s, field);
  if (!M) return -1;
  for (int l = s->geo.maxlevel; l > 0; l--) {
    const orc_lvl* Lc = &s->geo.lv[l - 1];
    const orc_lvl* Lf = &s->geo.lv[l];
    const double* f = M[l];
    double* c = M[l - 1];
    int Xl = Lf->nx - 1, Yl = Lf->ny - 1, Zl = Lf->nz - 1;
    long fsy = Lf->nx, fsz = (long)Lf->nx * Lf->ny;
#define MF(a, b, cc) f[(a) + (long)(b) * fsy + (long)(cc) * fsz]
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#pragma omp parallel for schedule(static)
    for (int ic = 0; ic < Lc->nx; ic++)
      for (int jc = 0; jc < Lc->ny; jc++)
        for (int kc = 0; kc < Lc->nz; kc++) {
          int x = 2 * ic, y = 2 * jc, z = 2 * kc;
          int xm = MAX(x - 1, 0), xp = MIN(x + 1, Xl), ym = MAX(y - 1, 0), yp = MIN(y + 1, Yl);
          int zm = MAX(z - 1, 0), zp = MIN(z + 1, Zl);
          double v[27] = {MF(xm, ym, zm), MF(xm, ym, zp), MF(xm, yp, zm), MF(xm, yp, zp), MF(xp, ym, zm),
                          MF(xp, ym, zp), MF(xp, yp, zm), MF(xp, yp, zp), MF(xm, ym, z),  MF(xm, yp, z),
                          MF(xp, ym, z),  MF(xp, yp, z),  MF(xm, y, zm),  MF(xm, y, zp),  MF(xp, y, zm),
                          MF(xp, y, zp),  MF(x, ym, zm),  MF(x, ym, zp),  MF(x, yp, zm),  MF(x, yp, zp),
                          MF(x, y, zm),   MF(x, y, zp),   MF(x, ym, z),   MF(x, yp, z),   MF(xm, y, z),
                          MF(xp, y, z),   MF(x, y, z)};
          double sv = v[0], sr = 1. / v[0];
          for (int q = 1; q < 27; ++q) {
            sv = sv + v[q];
            sr = sr + 1. / v[q];
          }
          double mv = 1.0 / 27.0 * sv;
          double mr = 27.0 / sr;
          c[ic + (long)jc * Lc->nx + (long)kc * Lc->nx * Lc->ny] = 0.5 * (0.5 * (mv + mr) + sqrt(mv * mr));
        }
#undef MF
#undef MAX
#undef MIN
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* history, right-hand side, reductions                                      */
/* ------------------------------------------------------------------------- */

/* strain_history (strain_history.cpp:162-210): H_e = max(H_e, 1/8 sum_g [phi+(s*eps_g) - gc_g/(2 lc)]). */
void orc_strain_history(orc_state* s, double lc, double u_proportion) {
  int l = s->geo.maxlevel;
  const orc_lvl* L = &s->geo.lv[l];
  shp sh;
  shape_init(&sh, L->hx, L->hy, L->hz);
  long N = lvl_n(L), off[8];
  node_offsets(L, off);
#pragma omp parallel for schedule(static)
  for (int k = 0; k <= L->nz - 2; k++)
    for (int j = 0; j <= L->ny - 2; j++)
      for (int i = 0; i <= L->nx - 2; i++) {
        long e = i + (long)j * L->nx + (long)k * L->nx * L->ny;
        double tmp = 0., eps[3][3];
        for (int g = 0; g < 8; g++) {
          double K_g = gpmp(s->bulK[l], e, off, sh.N[g]);
          double G_g = gpmp(s->G[l], e, off, sh.N[g]);
          double gc_g = gpmp(s->gc[l], e, off, sh.N[g]);
          strain_gp(&sh, s->u[l], N, e, off, g, eps);
          for (int c = 0; c < 3; c++)
            for (int m = 0; m < 3; m++) eps[c][m] = u_proportion * eps[c][m];
          tmp += phi_pos(K_g, G_g, eps) - 0.5 * gc_g / lc;
        }
        double H_tmp = 0.125 * tmp;
        if (s->H[l][e] < H_tmp) s->H[l][e] = H_tmp;
      }
}

/* fd_h (phase_field_right_hand_side.cpp:14-47): fd = sum_e 2 H_e wg sum_g N_g, sequential scatter. */
void orc_fd_h(orc_state* s, int l) {
  const orc_lvl* L = &s->geo.lv[l];
  shp sh;
  shape_init(&sh, L->hx, L->hy, L->hz);
  long N = lvl_n(L), off[8];
  node_offsets(L, off);
  double* fd = s->fd[l];
  const double* H = s->H[l];
  memset(fd, 0, sizeof(double) * N);
  for (int k = 0; k <= L->nz - 2; k++)
    for (int j = 0; j <= L->ny - 2; j++)
      for (int i = 0; i <= L->nx - 2; i++) {
        long e = i + (long)j * L->nx + (long)k * L->nx * L->ny;
        for (int tf = 0; tf < 8; tf++) {
          double v = 0.0;
          for (int g = 0; g < 8; g++) v += sh.wg * 2.0 * H[e] * sh.N[g][tf];
          fd[e + off[tf]] += v;
        }
      }
}

/* delta_d_max / d_max (phase_field_max_search.cpp:17-53); both start from 0. */
double orc_delta_d_max(orc_state* s) {
  int l = s->geo.maxlevel;
  long N = lvl_n(&s->geo.lv[l]);
  double m = 0.0;
  for (long i = 0; i < N; ++i)
    if (m < (s->d[l][i] - s->d_old[i])) m = s->d[l][i] - s->d_old[i];
  return m;
}
double orc_d_max(orc_state* s) {
  int l = s->geo.maxlevel;
  long N = lvl_n(&s->geo.lv[l]);
  double m = 0.0;
  for (long i = 0; i < N; ++i)
    if (m < s->d[l][i]) m = s->d[l][i];
  return m;
}

/* U_e (strain_history.cpp:86-131): min over elements and Gauss points of sqrt(phi_c / W). */
double orc_U_e(orc_state* s, double lc) {
  int l = s->geo.maxlevel;
  const orc_lvl* L = &s->geo.lv[l];
  shp sh;
  shape_init(&sh, L->hx, L->hy, L->hz);
  long N = lvl_n(L), off[8];
  node_offsets(L, off);
  double Ue = 1e10;
  for (int i = 0; i <= L->nx - 2; i++)
    for (int j = 0; j <= L->ny - 2; j++)
      for (int k = 0; k <= L->nz - 2; k++) {
        long e = i + (long)j * L->nx + (long)k * L->nx * L->ny;
        for (int g = 0; g < 8; g++) {
          double eps[3][3], sig[3][3];
          double K_g = gpmp(s->bulK[l], e, off, sh.N[g]);
          double G_g = gpmp(s->G[l], e, off, sh.N[g]);
          double gc_g = gpmp(s->gc[l], e, off, sh.N[g]);
          strain_gp(&sh, s->u[l], N, e, off, g, eps);
          double tr = trace3(eps);
          stress_gp(sig, eps, K_g, G_g, tr);
          double W0 = 0.;
          for (int c = 0; c < 3; c++)
            for (int m = 0; m < 3; m++) W0 += 0.5 * sig[c][m] * eps[c][m];
          double phi_c = 0.5 * gc_g / lc;
          double ut = sqrt(phi_c / W0);
          if (ut < Ue) Ue = ut;
        }
      }
  return Ue;
}

/* externe_force_nodal (mechanical_right_hnd.cpp:18-38): reactions into fu. */
void orc_externe_force_nodal(orc_state* s, double Ut, double small_k) {
  int l = s->geo.maxlevel;
  const orc_lvl* L = &s->geo.lv[l];
  long N = lvl_n(L);
  double* Fi = malloc(sizeof(double) * 3 * N);
  bc_apply(s, l, s->u[l], NULL, 0, Ut);
  orc_internal_force(L, 1, s->u[l], s->choice[l], s->bulK[l], s->G[l], s->d[l], s->Ke[l], s->Ge[l], small_k, Fi);
  bc_apply(s, l, s->fu[l], Fi, 1, 0.0);
  free(Fi);
}

/* externe_force_sum (mechanical_right_hnd.cpp:40-59): sum of fu_z over the top node plane. */
double orc_externe_force_sum(orc_state* s) {
  int l = s->geo.maxlevel;
  const orc_lvl* L = &s->geo.lv[l];
  long N = lvl_n(L), plane = (long)L->nx * L->ny;
  const double* fz = s->fu[l] + 2 * N;
  double ss = 0.0;
  for (long i = 0; i < plane; ++i) ss += fz[(long)(L->nz - 1) * plane + i];
  return ss;
}

/* initial_crack (strain_history.cpp:30-70); defined but never called by the reference. */
void orc_initial_crack(orc_state* s, double H_crack, int l) {
  const orc_lvl* L = &s->geo.lv[l];
  const orc_lvl* Lmax = &s->geo.lv[s->geo.maxlevel];
  const double* B = s->geo.box;
  for (int k = 0; k <= L->nz - 1; k++) {
    double z = B[4] + k * L->hz;
    for (int j = 0; j <= L->ny - 1; j++) {
      double y = B[2] + j * L->hy;
      for (int i = 0; i <= L->nx - 1; i++) {
        double x = B[0] + i * L->hx;
        if (z == 0.5 * (B[4] + B[5]) || z == 0.5 * (B[4] + B[5]) - Lmax->hz)
          if (y != B[3] || x != B[1]) s->H[l][i + (long)j * L->nx + (long)k * L->nx * L->ny] = H_crack;
      }
    }
  }
}

int orc_solution_injection(orc_state* s, int field, int comp, int lf) {
  double* f = array_of(s, field, lf, comp);
  double* c = array_of(s, field, lf - 1, comp);
  if (!f || !c) return -1;
  orc_injection(&s->geo.lv[lf - 1], &s->geo.lv[lf], f, c);
  return 0;
}
int orc_coarsen_f_standard(orc_state* s, int fc_field, int rf_field, int fic_field, int comp, int lf) {
  double* fc = array_of(s, fc_field, lf - 1, comp);
  double* rf = array_of(s, rf_field, lf, comp);
  double* fic = array_of(s, fic_field, lf - 1, comp);
  if (!fc || !rf || !fic) return -1;
  orc_restrict(&s->geo.lv[lf - 1], &s->geo.lv[lf], rf, fic, fc);
  return 0;
}
int orc_refine_standard(orc_state* s, int uf_field, int uc_field, int ucold_field, int comp, int lf) {
  double* uf = array_of(s, uf_field, lf, comp);
  double* uc = array_of(s, uc_field, lf - 1, comp);
  double* uo = array_of(s, ucold_field, lf - 1, comp);
  if (!uf || !uc || !uo) return -1;
  orc_prolong(&s->geo.lv[lf - 1], &s->geo.lv[lf], uc, uo, uf);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* solve drivers                                                             */
/* ------------------------------------------------------------------------- */

/* u_entire (mechanical_displacement.cpp:25-115); mech_tol is the squared-ratio test (1e-6 there).
 * Returns the V-cycles run (-1 on a zero diagonal); *iters = finest-level smoother iterations. */
int orc_u_entire(orc_state* s, const int* mg5, double small_k, double Ut, int t, double* f_norm, int* iters,
                 double mech_tol) {
  int Lm = s->geo.maxlevel;
  long N = lvl_n(&s->geo.lv[Lm]);
  int ncy = mg5[4];
  orc_mp_choice(s);
  memset(s->Ke[Lm], 0, sizeof(double) * N);
  memset(s->Ge[Lm], 0, sizeof(double) * N);
  orc_mp_all_element(s, small_k);
  orc_vr_all_level(s, ORC_KE);
  orc_vr_all_level(s, ORC_GE);
  double r_norm = orc_initial_residual_u(s, Lm, small_k);
  double rel = 1.0;
  if (t >= 1 && *f_norm != 0) rel = r_norm / *f_norm;
  int cycles = 0, fin = 0;
  /* finest-level smoother iterations per cycle */
  int per_cycle = (Lm == 0) ? mg5[0] : mg5[1] + mg5[2];
  for (int j = 1; j <= ncy; j++) {
    if (rel > mech_tol) {
      if (orc_cycle_u(s, Lm, mg5, small_k, Ut, t, f_norm) < 0) return -1;
      cycles++;
      fin += per_cycle;
      bc_apply(s, Lm, s->ru[Lm], NULL, 2, 0.0);
      r_norm = 0.0;
      for (int di = 0; di < 3; ++di) r_norm += dot_n(s->ru[Lm] + di * N, s->ru[Lm] + di * N, N);
      rel = r_norm / *f_norm;
    }
    if (rel <= mech_tol) break;
  }
  orc_externe_force_nodal(s, Ut, small_k);
  if (iters) *iters = fin;
  return cycles;
}

/* phase_field (phase_field.cpp:15-57); pf_tol is both the absolute and the relative squared test. */
int orc_phase_field(orc_state* s, const int* mg5, double lc, int t, double* fd_norm, int* iters, double pf_tol) {
  int Lm = s->geo.maxlevel;
  long N = lvl_n(&s->geo.lv[Lm]);
  int ncy = mg5[4];
  double r_norm = orc_initial_residual_d(s, Lm, lc);
  double sres = 1.0;
  int cycles = 0, fin = 0;
  int per_cycle = (Lm == 0) ? mg5[0] : mg5[1] + mg5[2] * mg5[2];
  for (int j = 1; j <= ncy; j++) {
    if (r_norm > pf_tol) {
      if (sres > pf_tol) {
        if (orc_cycle_d(s, Lm, mg5, lc, t, fd_norm) < 0) return -1;
        cycles++;
        fin += per_cycle;
      }
      r_norm = dot_n(s->R[Lm], s->R[Lm], N);
      sres = r_norm / *fd_norm;
      if (sres <= pf_tol) break;
    } else {
      break;
    }
  }
  if (iters) *iters = fin;
  return cycles;
}

/* findPosition (csv_reader.cpp:65-73). */
static int find_position(const int* gray, int ngray, int x) {
  for (int i = 0; i < ngray - 1; ++i)
    if (x >= gray[i] && x <= gray[i + 1]) return i;
  return -1;
}

/* image_MP (image_input.cpp:120-142) + coarse_VR for bulK, G, gc.  The gray-level interpolation
 * weight is an integer division in the reference (:135-137), reproduced here. */
int orc_image_material(orc_state* s, const unsigned char* image, const int* voxel_n, int ngray,
                       const int* gray, const double* E, const double* nu, const double* gcv,
                       double voxel_size) {
  int l = s->geo.maxlevel;
  const orc_lvl* L = &s->geo.lv[l];
  const int* roi = s->geo.roi;
  for (int k = 0; k < L->nz; k++)
    for (int j = 0; j < L->ny; j++)
      for (int i = 0; i < L->nx; i++) {
        long long x = roi[0] + i + (long long)voxel_n[0] * (roi[1] + j) +
                      (long long)voxel_n[0] * voxel_n[1] * (roi[2] + k);
        int gl = image[x];
        int p = find_position(gray, ngray, gl);
        if (p < 0) return -1;
        int q = (gl - gray[p]) / (gray[p + 1] - gray[p]);
        double Ev = E[p] + q * (E[p + 1] - E[p]);
        double nv = nu[p] + q * (nu[p + 1] - nu[p]);
        long n = i + (long)j * L->nx + (long)k * L->nx * L->ny;
        s->gc[l][n] = gcv[p] + q * (gcv[p + 1] - gcv[p]);
        Ev = voxel_size * Ev;
        s->bulK[l][n] = 1.0 / (3.0 * (1.0 - 2.0 * nv)) * Ev;
        s->G[l][n] = 1.0 / (2.0 * (1.0 + nv)) * Ev;
      }
  orc_coarse_vr(s, ORC_BULK);
  orc_coarse_vr(s, ORC_G);
  orc_coarse_vr(s, ORC_GC);
  return 0;
}

/* One staggered increment: the loop body of crack_propagation (crack_propagation.cpp:65-121) with its
 * constants as parameters (see oracle/ref_harness.cpp ref_step for the meaning of out[]). */
int orc_step(orc_state* s, int t, const int* mg_u, const int* mg_d, double small_k, double lc,
             double voxel_size, double ut0, double dU, double dU_factor, double mech_tol, double pf_tol,
             double* out) {
  const double U_unit = 1.0;
  int Lm = s->geo.maxlevel;
  long N = lvl_n(&s->geo.lv[Lm]);
  int mech_it = 0, pf_it = 0;
  int mech_cy = orc_u_entire(s, mg_u, small_k, U_unit, t, &s->f_norm, &mech_it, mech_tol);
  if (mech_cy < 0) return -1;
  if (t == 0) {
    if (ut0 <= 0.0) {
      s->Ue = orc_U_e(s, lc);
      s->Ut = s->Ue;
      s->dU = dU_factor * s->Ue;
    } else {
      s->Ue = ut0;
      s->Ut = ut0;
      s->dU = dU;
    }
    s->uprop = s->Ut / U_unit;
  }
  orc_strain_history(s, lc, s->uprop);
  orc_voigt_all_level(s, ORC_H);
  for (int l = Lm; l >= 0; l--) orc_fd_h(s, l);
  int pf_cy = orc_phase_field(s, mg_d, lc, t, &s->fd_norm, &pf_it, pf_tol);
  if (pf_cy < 0) return -1;
  double dd = orc_delta_d_max(s);
  memcpy(s->d_old, s->d[Lm], sizeof(double) * N);
  double FeW = orc_externe_force_sum(s) * voxel_size;
  double dmax = orc_d_max(s);
  double Ut_now = s->Ut;
  s->Ut = s->Ut + s->dU;
  s->uprop = s->Ut / U_unit;
  out[0] = Ut_now;
  out[1] = s->uprop * FeW;
  out[2] = dd;
  out[3] = dmax;
  out[4] = mech_cy;
  out[5] = pf_cy;
  out[6] = mech_it;
  out[7] = pf_it;
  return 0;
}
