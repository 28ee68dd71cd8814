/*
 * C-ABI harness over the REFERENCE HPCrack implementation, compiled from the
 * reference's own sources (see oracle/Makefile) into oracle/_ref/libhpcref.so.
 *
 * Test infrastructure only: it is the "reference" oracle that pins the plain-C
 * restatement (oracle/hpc_oracle.c) and serves as the CPU baseline arm of
 * bench.py.  Nothing in the product library links or calls it.
 *
 * Every entry point builds the reference's own objects (Stack, MPI_Setting,
 * mg / mgvec / grid) and calls the reference's functions on them; arrays cross
 * the boundary as plain x-fastest double / short buffers, the same layout as
 * grid<T>::operator() (include/grid.h:83-91).
 */
#include <unistd.h>
#include <fcntl.h>
#include <omp.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <iostream>

#include "configuration.h"
#include "initialization.h"
#include "mpi_environment_setup.h"
#include "mg.h"
#include "mgvec.h"
#include "grid2d.h"
#include "shape_function.h"
#include "mechanical_pcg.h"
#include "phase_field_pcg.h"
#include "mechanical_multigrid.h"
#include "phase_field_multigrid.h"
#include "mechanical_displacement.h"
#include "phase_field.h"
#include "multigrid_intergrid.h"
#include "material_selection.h"
#include "material_coarse_element.h"
#include "strain_history.h"
#include "phase_field_right_hand_side.h"
#include "phase_field_max_search.h"
#include "mechanical_right_hand_side.h"
#include "boundary_conditions.h"
#include "image_input.h"
#include "pcg_utilities.h"
#include "write_read_history.h"
#include "vtk_output.h"

namespace {

enum Field {
  F_BULK = 0, F_G = 1, F_GC = 2, F_D = 3, F_H = 4, F_FD = 5, F_KE = 6, F_GE = 7,
  F_R = 8, F_DOLD = 9, F_DOLDF = 10,
  F_U = 16, F_FU = 17, F_RU = 18, F_UOLD = 19,
  F_CHOICE = 32
};

struct RefCtx {
  Stack U;
  MPI_Setting M;
  Parameters para;
  int maxlevel;
  mgdouble *bulK, *G, *gc, *d, *H, *fd, *Ke, *Ge, *R, *dold;
  mgvecdouble *u, *fu, *ru, *uold;
  mgshort* choice;
  griddouble* d_old;  // finest-level d of the previous increment (crack_propagation.cpp:45)
  // staggered-loop state (crack_propagation.cpp:32-39)
  double f_norm, fd_norm, Ue, Ut, delta_U, u_proportion;
};

bool g_quiet = true;
std::string g_last_out;

// Runs fn with fd 1 redirected to a temporary file; the text is kept in g_last_out.
template <class Fn>
void captured(Fn fn) {
  std::cout.flush();
  fflush(stdout);
  char path[] = "/tmp/hpcref_outXXXXXX";
  int tmp = mkstemp(path);
  int saved = dup(1);
  dup2(tmp, 1);
  fn();
  std::cout.flush();
  fflush(stdout);
  dup2(saved, 1);
  close(saved);
  g_last_out.clear();
  lseek(tmp, 0, SEEK_SET);
  char buf[65536];
  ssize_t n;
  while ((n = read(tmp, buf, sizeof buf)) > 0) g_last_out.append(buf, (size_t)n);
  close(tmp);
  unlink(path);
  if (!g_quiet) { fwrite(g_last_out.data(), 1, g_last_out.size(), stdout); fflush(stdout); }
}

int count_occurrences(const std::string& s, const char* pat) {
  int c = 0;
  size_t pos = 0, L = strlen(pat);
  while ((pos = s.find(pat, pos)) != std::string::npos) { ++c; pos += L; }
  return c;
}

mgdouble* scalar_field(RefCtx* c, int f) {
  switch (f) {
    case F_BULK: return c->bulK;
    case F_G: return c->G;
    case F_GC: return c->gc;
    case F_D: return c->d;
    case F_H: return c->H;
    case F_FD: return c->fd;
    case F_KE: return c->Ke;
    case F_GE: return c->Ge;
    case F_R: return c->R;
    case F_DOLD: return c->dold;
    default: return nullptr;
  }
}
mgvecdouble* vector_field(RefCtx* c, int f) {
  switch (f) {
    case F_U: return c->u;
    case F_FU: return c->fu;
    case F_RU: return c->ru;
    case F_UOLD: return c->uold;
    default: return nullptr;
  }
}
griddouble* grid_of(RefCtx* c, int f, int level, int comp) {
  if (f == F_DOLDF) return c->d_old;
  if (mgdouble* m = scalar_field(c, f)) {
    if (level < 0 || level >= m->nbl()) return nullptr;
    return &m->getLevel(level);
  }
  if (mgvecdouble* v = vector_field(c, f)) {
    if (level < 0 || level >= v->nbl() || comp < 0 || comp > 2) return nullptr;
    return &v->getLevel(level).getgrid(comp);
  }
  return nullptr;
}

struct Shape {
  grid2d N;
  griddouble DN;
  double wg;
  Shape(const Level* L) : N(8, 8), DN(std::vector<size_t>{3, 8, 8}) {
    Dshape_function(N, DN, L->hx, L->hy, L->hz);
    wg = 0.125 * L->hx * L->hy * L->hz;
  }
};

}  // namespace

extern "C" {

void ref_set_quiet(int q) { g_quiet = q != 0; }
void ref_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }
int ref_get_threads(void) { return omp_get_max_threads(); }

/* Builds the hierarchy exactly as main.cpp:70-78 does for one rank:
 * input_setting (image_input.cpp:21-27) then initialize (initialization.cpp:19-134). */
void* ref_ctx_create(int maxlevel, const int* element_nb, const double* x_start, const int* roi_start) {
  RefCtx* c = new RefCtx();
  c->maxlevel = maxlevel;
  c->para.D = 3;
  c->para.np = {1, 1, 1};
  c->para.X_start = {x_start[0], x_start[1], x_start[2]};
  c->para.element_nb = {element_nb[0], element_nb[1], element_nb[2]};
  c->para.IDM.coefxa = roi_start[0];
  c->para.IDM.coefya = roi_start[1];
  c->para.IDM.coefza = roi_start[2];
  Set_MPI(&c->M, c->para.np);
  input_setting(c->para.IDM, c->para.element_nb, maxlevel);
  captured([&] { initialize(&c->U, c->para, c->M, maxlevel); });
  Stack* U = &c->U;
  c->bulK = new mgdouble(U, maxlevel);
  c->G = new mgdouble(U, maxlevel);
  c->gc = new mgdouble(U, maxlevel);
  c->d = new mgdouble(U, maxlevel);
  c->H = new mgdouble(U, maxlevel);
  c->fd = new mgdouble(U, maxlevel);
  c->Ke = new mgdouble(U, maxlevel);
  c->Ge = new mgdouble(U, maxlevel);
  c->R = new mgdouble(U, maxlevel);
  c->dold = new mgdouble(U, maxlevel);
  c->u = new mgvecdouble(U, maxlevel, 3);
  c->fu = new mgvecdouble(U, maxlevel, 3);
  c->ru = new mgvecdouble(U, maxlevel, 3);
  c->uold = new mgvecdouble(U, maxlevel, 3);
  c->choice = new mgshort(U, maxlevel);
  c->d_old = new griddouble(c->d->getLevel(maxlevel).axis());
  c->f_norm = c->fd_norm = c->Ue = c->Ut = c->delta_U = c->u_proportion = 0.0;
  return c;
}

void ref_ctx_destroy(void* h) {
  RefCtx* c = (RefCtx*)h;
  if (!c) return;
  delete c->bulK; delete c->G; delete c->gc; delete c->d; delete c->H; delete c->fd;
  delete c->Ke; delete c->Ge; delete c->R; delete c->dold;
  delete c->u; delete c->fu; delete c->ru; delete c->uold;
  delete c->choice; delete c->d_old;
  finalize(&c->U);
  delete c;
}

/* Level geometry as initialize() produced it: n[3] nodes, h[3] spacings, ii/jj/kk elements. */
void ref_level_info(void* h, int level, int* n3, double* h3, long* e3) {
  RefCtx* c = (RefCtx*)h;
  Level* L = c->U.Ll + level;
  n3[0] = L->nbcolox; n3[1] = L->nbcoloy; n3[2] = L->nbcoloz;
  h3[0] = L->hx; h3[1] = L->hy; h3[2] = L->hz;
  e3[0] = L->ii; e3[1] = L->jj; e3[2] = L->kk;
}
void ref_domain(void* h, double* box6) {
  RefCtx* c = (RefCtx*)h;
  box6[0] = c->U.xa; box6[1] = c->U.xb; box6[2] = c->U.ya;
  box6[3] = c->U.yb; box6[4] = c->U.za; box6[5] = c->U.zb;
}

int ref_set(void* h, int field, int level, int comp, const double* src) {
  RefCtx* c = (RefCtx*)h;
  griddouble* g = grid_of(c, field, level, comp);
  if (!g) return -1;
  size_t n = g->size();
  for (size_t i = 0; i < n; ++i) (*g)[i] = src[i];
  return 0;
}
int ref_get(void* h, int field, int level, int comp, double* dst) {
  RefCtx* c = (RefCtx*)h;
  griddouble* g = grid_of(c, field, level, comp);
  if (!g) return -1;
  size_t n = g->size();
  for (size_t i = 0; i < n; ++i) dst[i] = (*g)[i];
  return 0;
}
int ref_set_choice(void* h, int level, const short* src) {
  RefCtx* c = (RefCtx*)h;
  gridshort& g = c->choice->getLevel(level);
  for (size_t i = 0; i < g.size(); ++i) g[i] = src[i];
  return 0;
}
int ref_get_choice(void* h, int level, short* dst) {
  RefCtx* c = (RefCtx*)h;
  gridshort& g = c->choice->getLevel(level);
  for (size_t i = 0; i < g.size(); ++i) dst[i] = g[i];
  return 0;
}

/* ---------------- operators (mechanical_pcg.cpp, phase_field_pcg.cpp) ---------------- */

/* Fi = K(d) u on one level: Internal_Force (mechanical_pcg.cpp:174-191). */
int ref_internal_force(void* h, int level, int src, int dst, double small_k) {
  RefCtx* c = (RefCtx*)h;
  mgvecdouble* s = vector_field(c, src);
  mgvecdouble* o = vector_field(c, dst);
  if (!s || !o || s == o) return -1;
  Shape sh(c->U.Ll + level);
  Internal_Force(&c->U, o->getLevel(level), s->getLevel(level), c->choice->getLevel(level),
                 c->bulK->getLevel(level), c->G->getLevel(level), c->d->getLevel(level),
                 c->Ke->getLevel(level), c->Ge->getLevel(level), sh.DN, sh.N, sh.wg, level, small_k);
  return 0;
}

/* diag(K(d)) on one level: PreM_u (mechanical_pcg.cpp:102-112) on a zeroed output. */
int ref_prem_u(void* h, int level, int dst, double small_k) {
  RefCtx* c = (RefCtx*)h;
  mgvecdouble* o = vector_field(c, dst);
  if (!o) return -1;
  for (int di = 0; di < 3; ++di) o->getLevel(level).getgrid(di).Assign_zero();
  Shape sh(c->U.Ll + level);
  PreM_u(&c->U, o->getLevel(level), c->choice->getLevel(level), c->bulK->getLevel(level),
         c->G->getLevel(level), c->d->getLevel(level), c->Ke->getLevel(level), c->Ge->getLevel(level),
         sh.DN, sh.N, sh.wg, level, small_k);
  return 0;
}

/* Fi = A_d x on one level: Fld (phase_field_pcg.cpp:93-103). */
int ref_fld(void* h, int level, int src, int dst, double lc) {
  RefCtx* c = (RefCtx*)h;
  mgdouble* s = scalar_field(c, src);
  mgdouble* o = scalar_field(c, dst);
  if (!s || !o || s == o) return -1;
  Shape sh(c->U.Ll + level);
  Fld(o->getLevel(level), s->getLevel(level), c->H->getLevel(level), c->gc->getLevel(level), sh.DN,
      sh.N, lc, sh.wg);
  return 0;
}

/* diag(A_d): Precondition_M (phase_field_pcg.cpp:49-59). */
int ref_precondition_m(void* h, int level, int dst, double lc) {
  RefCtx* c = (RefCtx*)h;
  mgdouble* o = scalar_field(c, dst);
  if (!o) return -1;
  Shape sh(c->U.Ll + level);
  Precondition_M(o->getLevel(level), c->H->getLevel(level), c->gc->getLevel(level), sh.DN, sh.N, lc,
                 sh.wg);
  return 0;
}

double ref_initial_residual_u(void* h, int level, double small_k) {
  RefCtx* c = (RefCtx*)h;
  double r = 0.0;
  captured([&] {
    r = Initial_residual_u(&c->U, c->ru->getLevel(level), c->u->getLevel(level),
                           c->fu->getLevel(level), c->choice->getLevel(level), c->bulK->getLevel(level),
                           c->G->getLevel(level), c->d->getLevel(level), c->Ke->getLevel(level),
                           c->Ge->getLevel(level), c->M, level, small_k);
  });
  return r;
}

/* One pcg_u call (mechanical_pcg.cpp:223-330) on the harness's u / ru / fu of a level. */
int ref_pcg_u(void* h, int level, double small_k, double Ut, int nb_relax, int t, double* f_norm) {
  RefCtx* c = (RefCtx*)h;
  captured([&] {
    pcg_u(&c->U, c->u->getLevel(level), c->ru->getLevel(level), c->fu->getLevel(level),
          c->choice->getLevel(level), c->bulK->getLevel(level), c->G->getLevel(level),
          c->d->getLevel(level), c->Ke->getLevel(level), c->Ge->getLevel(level), c->M, level, small_k,
          Ut, nb_relax, t, *f_norm);
  });
  return count_occurrences(g_last_out, " Ru =");
}

double ref_initial_residual_d(void* h, int level, double lc) {
  RefCtx* c = (RefCtx*)h;
  return initial_residual(&c->U, c->R->getLevel(level), c->d->getLevel(level), c->fd->getLevel(level),
                          c->H->getLevel(level), c->gc->getLevel(level), level, lc, c->M);
}

/* One pcg_d call (phase_field_pcg.cpp:133-214). */
int ref_pcg_d(void* h, int level, double lc, int nb_relax, int t, double* fd_norm) {
  RefCtx* c = (RefCtx*)h;
  captured([&] {
    pcg_d(&c->U, c->d->getLevel(level), c->fd->getLevel(level), c->R->getLevel(level),
          c->H->getLevel(level), c->gc->getLevel(level), c->M, level, lc, nb_relax, t, *fd_norm);
  });
  return count_occurrences(g_last_out, " Rd =");
}

/* One FAS cycle from `level` down (mechanical_multigrid.cpp:18-54). Returns smoother iterations run. */
int ref_cycle_u(void* h, int level, const int* mg5, double small_k, double Ut, int t, double* f_norm) {
  RefCtx* c = (RefCtx*)h;
  MG p{mg5[0], mg5[1], mg5[2], mg5[3], mg5[4]};
  captured([&] {
    cycle_u(&c->U, *c->u, *c->ru, *c->fu, *c->uold, *c->choice, *c->bulK, *c->G, *c->d, *c->Ke, *c->Ge,
            level, p, c->M, 0, 1, small_k, Ut, t, *f_norm);
  });
  return count_occurrences(g_last_out, " Ru =");
}

int ref_cycle_d(void* h, int level, const int* mg5, double lc, int t, double* fd_norm) {
  RefCtx* c = (RefCtx*)h;
  MG p{mg5[0], mg5[1], mg5[2], mg5[3], mg5[4]};
  captured([&] {
    cycle_d(&c->U, *c->d, *c->fd, *c->dold, *c->H, *c->gc, *c->R, level, lc, p, c->M, 0, 1, t,
            *fd_norm);
  });
  return count_occurrences(g_last_out, " Rd =");
}

/* The whole mechanical solve u_entire (mechanical_displacement.cpp:25-115).
 * Returns the number of V-cycles run; *iters gets the finest-level smoother iterations. */
int ref_u_entire(void* h, const int* mg5, double small_k, double Ut, int t, double* f_norm, int* iters) {
  RefCtx* c = (RefCtx*)h;
  MG p{mg5[0], mg5[1], mg5[2], mg5[3], mg5[4]};
  captured([&] {
    u_entire(&c->U, *c->u, *c->fu, *c->bulK, *c->G, *c->d, c->M, p, 0, 1, small_k, Ut, t, *f_norm);
  });
  if (iters) {
    char pat[32];
    snprintf(pat, sizeof pat, "Level %d Ru =", c->maxlevel);
    *iters = count_occurrences(g_last_out, pat);
  }
  return count_occurrences(g_last_out, ",Cycle=");
}

/* The whole phase-field solve (phase_field.cpp:15-57). Returns V-cycles run. */
int ref_phase_field(void* h, const int* mg5, double lc, int t, double* fd_norm, int* iters) {
  RefCtx* c = (RefCtx*)h;
  MG p{mg5[0], mg5[1], mg5[2], mg5[3], mg5[4]};
  captured([&] { phase_field(&c->U, *c->d, *c->fd, *c->H, *c->gc, c->M, lc, p, 0, 1, t, *fd_norm); });
  if (iters) {
    char pat[32];
    snprintf(pat, sizeof pat, "Level %d Rd =", c->maxlevel);
    *iters = count_occurrences(g_last_out, pat);
  }
  return count_occurrences(g_last_out, ",Cycle=");
}

/* u_entire (mechanical_displacement.cpp:25-115) with its stopping threshold as a parameter (the
 * reference hard-codes |r|^2/|f|^2 <= 1e-6 at :88,102).  The driver makes the reference's own calls
 * in u_entire's order on work containers created the way u_entire creates them (fresh regime grid,
 * element moduli, uold, ru): MP_choice, MP_all_element, VR_all_level x2, Initial_residual_u, then
 * cycle_u + Dirichlet_residual_u + grid_norm per cycle until the threshold, then
 * externe_force_nodal.  With tol = 1e-6 it reproduces u_entire; smaller tol is the tolerance of the
 * benchmark configurations (|r|/|f| <= 1e-8 is tol = 1e-16). */
int ref_u_entire_tol(void* h, const int* mg5, double small_k, double Ut, int t, double* f_norm, int* iters,
                     double tol) {
  RefCtx* c = (RefCtx*)h;
  Stack* U = &c->U;
  const int L = U->maxlevel;
  MG p{mg5[0], mg5[1], mg5[2], mg5[3], mg5[4]};
  int cycles = 0;
  captured([&] {
    mgvecdouble uold(U, L - 1, 3);
    mgvecdouble ru(U, L, 3);
    mgshort choice(U, L);
    mgdouble Ke(U, L), Ge(U, L);
    MP_choice(U, choice, *c->u, *c->bulK, *c->G, *c->d);
    MP_all_element(U, c->u->getLevel(L), c->bulK->getLevel(L), c->G->getLevel(L), c->d->getLevel(L),
                   choice.getLevel(L), Ke.getLevel(L), Ge.getLevel(L), L, small_k);
    VR_all_level(Ke, c->M);
    VR_all_level(Ge, c->M);
    double rn = Initial_residual_u(U, ru.getLevel(L), c->u->getLevel(L), c->fu->getLevel(L), choice.getLevel(L),
                                   c->bulK->getLevel(L), c->G->getLevel(L), c->d->getLevel(L), Ke.getLevel(L),
                                   Ge.getLevel(L), c->M, L, small_k);
    double rel = (t >= 1 && *f_norm != 0) ? rn / *f_norm : 1.0;
    for (int j = 1; j <= p.ncy && rel > tol; ++j) {
      cycle_u(U, *c->u, ru, *c->fu, uold, choice, *c->bulK, *c->G, *c->d, Ke, Ge, L, p, c->M, 0, 1, small_k, Ut,
              t, *f_norm);
      Dirichlet_residual_u(U, ru.getLevel(L), c->M, L);
      rn = 0.0;
      for (int m = 0; m < 3; ++m) rn += grid_norm(ru.getLevel(L).getgrid(m), c->M);
      rel = rn / *f_norm;
      ++cycles;
    }
    externe_force_nodal(U, c->fu->getLevel(L), c->u->getLevel(L), choice.getLevel(L), c->bulK->getLevel(L),
                        c->G->getLevel(L), c->d->getLevel(L), Ke.getLevel(L), Ge.getLevel(L), c->M, L, Ut, small_k);
  });
  if (iters) {
    char pat[32];
    snprintf(pat, sizeof pat, "Level %d Ru =", L);
    *iters = count_occurrences(g_last_out, pat);
  }
  return cycles;
}

/* phase_field (phase_field.cpp:15-57) with its threshold as a parameter (1e-12 at :30,33,41 in the
 * reference): cycle_d until |R|^2 <= tol or |R|^2/|fd|^2 <= tol, on a fresh dold and R. */
int ref_phase_field_tol(void* h, const int* mg5, double lc, int t, double* fd_norm, int* iters, double tol) {
  RefCtx* c = (RefCtx*)h;
  Stack* U = &c->U;
  const int L = U->maxlevel;
  MG p{mg5[0], mg5[1], mg5[2], mg5[3], mg5[4]};
  int cycles = 0;
  captured([&] {
    mgdouble dold(U, L - 1);
    mgdouble R(U, L);
    double rn = initial_residual(U, R.getLevel(L), c->d->getLevel(L), c->fd->getLevel(L), c->H->getLevel(L),
                                 c->gc->getLevel(L), L, lc, c->M);
    double srel = 1.0;
    for (int j = 1; j <= p.ncy && rn > tol; ++j) {
      if (srel > tol) {
        cycle_d(U, *c->d, *c->fd, dold, *c->H, *c->gc, R, L, lc, p, c->M, 0, 1, t, *fd_norm);
        ++cycles;
      }
      rn = grid_norm(R.getLevel(L), c->M);
      srel = rn / *fd_norm;
      if (srel <= tol) break;
    }
  });
  if (iters) {
    char pat[32];
    snprintf(pat, sizeof pat, "Level %d Rd =", L);
    *iters = count_occurrences(g_last_out, pat);
  }
  return cycles;
}

/* ---------------- material / history kernels ---------------- */

/* MP_choice on a freshly zeroed field, as its only caller does (mechanical_displacement.cpp:33,38). */
void ref_mp_choice(void* h) {
  RefCtx* c = (RefCtx*)h;
  for (int l = 0; l <= c->maxlevel; ++l) {
    gridshort& g = c->choice->getLevel(l);
    for (size_t i = 0; i < g.size(); ++i) g[i] = 0;
  }
  MP_choice(&c->U, *c->choice, *c->u, *c->bulK, *c->G, *c->d);
}
void ref_mp_all_element(void* h, double small_k) {
  RefCtx* c = (RefCtx*)h;
  int L = c->maxlevel;
  MP_all_element(&c->U, c->u->getLevel(L), c->bulK->getLevel(L), c->G->getLevel(L), c->d->getLevel(L),
                 c->choice->getLevel(L), c->Ke->getLevel(L), c->Ge->getLevel(L), L, small_k);
}
int ref_vr_all_level(void* h, int field) {
  RefCtx* c = (RefCtx*)h;
  mgdouble* m = scalar_field(c, field);
  if (!m) return -1;
  VR_all_level(*m, c->M);
  return 0;
}
int ref_voigt_all_level(void* h, int field) {
  RefCtx* c = (RefCtx*)h;
  mgdouble* m = scalar_field(c, field);
  if (!m) return -1;
  Voigt_all_level(*m, c->M);
  return 0;
}
/* Nodal 27-point Voigt-Reuss-Hill of a material field to every coarse level (image_input.cpp:244-260). */
int ref_coarse_vr(void* h, int field) {
  RefCtx* c = (RefCtx*)h;
  mgdouble* m = scalar_field(c, field);
  if (!m) return -1;
  coarse_VR(*m, c->M);
  return 0;
}
void ref_strain_history(void* h, double lc, double u_proportion) {
  RefCtx* c = (RefCtx*)h;
  int L = c->maxlevel;
  strain_history(&c->U, c->H->getLevel(L), c->u->getLevel(L), c->bulK->getLevel(L), c->G->getLevel(L),
                 c->gc->getLevel(L), c->M, L, lc, u_proportion);
}
void ref_fd_h(void* h, int level) {
  RefCtx* c = (RefCtx*)h;
  fd_h(&c->U, c->fd->getLevel(level), c->H->getLevel(level), level);
}
double ref_delta_d_max(void* h) {
  RefCtx* c = (RefCtx*)h;
  return delta_d_max(c->d->getLevel(c->maxlevel), *c->d_old);
}
double ref_d_max(void* h) {
  RefCtx* c = (RefCtx*)h;
  return d_max(c->d->getLevel(c->maxlevel));
}
double ref_U_e(void* h, double lc) {
  RefCtx* c = (RefCtx*)h;
  int L = c->maxlevel;
  return U_e(&c->U, c->u->getLevel(L), c->bulK->getLevel(L), c->G->getLevel(L), c->gc->getLevel(L), L,
             lc, c->M);
}
void ref_externe_force_nodal(void* h, double Ut, double small_k) {
  RefCtx* c = (RefCtx*)h;
  int L = c->maxlevel;
  externe_force_nodal(&c->U, c->fu->getLevel(L), c->u->getLevel(L), c->choice->getLevel(L),
                      c->bulK->getLevel(L), c->G->getLevel(L), c->d->getLevel(L), c->Ke->getLevel(L),
                      c->Ge->getLevel(L), c->M, L, Ut, small_k);
}
double ref_externe_force_sum(void* h) {
  RefCtx* c = (RefCtx*)h;
  return externe_force_sum(c->fu->getLevel(c->maxlevel).getgrid(2), c->M);
}
void ref_initial_crack(void* h, double H_crack, int level) {
  RefCtx* c = (RefCtx*)h;
  initial_crack(&c->U, c->H->getLevel(level), c->M, H_crack, level);
}

/* ---------------- boundary conditions (boundary_conditions.cpp:20-154) ---------------- */

int ref_dirichlet_bd(void* h, int level, int field, double Ut) {
  RefCtx* c = (RefCtx*)h;
  mgvecdouble* v = vector_field(c, field);
  if (!v) return -1;
  Dirichlet_BD(&c->U, v->getLevel(level), c->M, level, Ut);
  return 0;
}
int ref_dirichlet_force(void* h, int level, int f_field, int fi_field) {
  RefCtx* c = (RefCtx*)h;
  mgvecdouble* f = vector_field(c, f_field);
  mgvecdouble* fi = vector_field(c, fi_field);
  if (!f || !fi) return -1;
  Dirichlet_force_u(&c->U, f->getLevel(level), fi->getLevel(level), c->M, level);
  return 0;
}
int ref_dirichlet_residual(void* h, int level, int field) {
  RefCtx* c = (RefCtx*)h;
  mgvecdouble* v = vector_field(c, field);
  if (!v) return -1;
  Dirichlet_residual_u(&c->U, v->getLevel(level), c->M, level);
  return 0;
}

/* ---------------- inter-grid transfers (multigrid_intergrid.cpp) ---------------- */

/* Scalar transfers between levels lf and lf-1 of one field. */
int ref_solution_injection(void* h, int field, int comp, int lf) {
  RefCtx* c = (RefCtx*)h;
  griddouble* f = grid_of(c, field, lf, comp);
  griddouble* co = grid_of(c, field, lf - 1, comp);
  if (!f || !co) return -1;
  solution_injection(*co, *f, c->M);
  return 0;
}
/* fc = Fic + full-weighting(rf) (coarsen_f_standard_routine, :124-342); fields at levels lf-1 / lf. */
int ref_coarsen_f_standard(void* h, int fc_field, int rf_field, int fic_field, int comp, int lf) {
  RefCtx* c = (RefCtx*)h;
  griddouble* fc = grid_of(c, fc_field, lf - 1, comp);
  griddouble* rf = grid_of(c, rf_field, lf, comp);
  griddouble* fic = grid_of(c, fic_field, lf - 1, comp);
  if (!fc || !rf || !fic) return -1;
  coarsen_f_standard_routine(*fc, *rf, *fic, c->M);
  return 0;
}
/* uf += P(uc - ucold) (refine_standard_routine, :416-520). */
int ref_refine_standard(void* h, int uf_field, int uc_field, int ucold_field, int comp, int lf) {
  RefCtx* c = (RefCtx*)h;
  griddouble* uf = grid_of(c, uf_field, lf, comp);
  griddouble* uc = grid_of(c, uc_field, lf - 1, comp);
  griddouble* uo = grid_of(c, ucold_field, lf - 1, comp);
  if (!uf || !uc || !uo) return -1;
  refine_standard_routine(*uf, *uc, *uo, c->M);
  return 0;
}

/* ---------------- input path (image_input.cpp, csv_reader.cpp) ---------------- */

/* image_MP + coarse_VR for bulK, G, gc (image_input.cpp:120-282).  The reference reads the CSV from
 * the fixed relative path data/Material_Property.csv (csv_reader.cpp:22), so the working directory is
 * switched to `workdir` for the call.  voxel_n[3] = image size; the ROI start is the context's. */
int ref_input_total(void* h, const char* workdir, const char* raw_path, const int* voxel_n,
                    double voxel_size) {
  RefCtx* c = (RefCtx*)h;
  c->para.IDM.voxelnx = voxel_n[0];
  c->para.IDM.voxelny = voxel_n[1];
  c->para.IDM.voxelnz = voxel_n[2];
  c->para.IMGname = raw_path;
  c->para.voxel_size = voxel_size;
  char cwd[4096];
  if (!getcwd(cwd, sizeof cwd)) return -1;
  if (chdir(workdir) != 0) return -2;
  captured([&] { input_total(&c->U, *c->bulK, *c->G, *c->gc, c->M, c->para); });
  if (chdir(cwd) != 0) return -3;
  return 0;
}

/* ---------------- one staggered increment (crack_propagation.cpp:65-121) ----------------
 * The loop body of crack_propagation with its hard-coded constants made parameters:
 * small_k (:32), U_unit (:37), the load schedule (:71-80, :112; ut0 <= 0 selects the reference's
 * Ue-based schedule Ut = Ue + t*dU_factor*Ue, otherwise Ut = ut0 + t*dU), mechanical /
 * phase-field tolerances are the reference's (compiled into u_entire / phase_field).
 * out[8] = {Ut, FeW*u_proportion, delta_d_max, d_max, mech cycles, pf cycles, mech finest iters,
 *           pf finest iters}. */
int ref_step(void* h, int t, const int* mg_u, const int* mg_d, double small_k, double lc, double voxel_size,
             double ut0, double dU, double dU_factor, double mech_tol, double pf_tol, double* out) {
  RefCtx* c = (RefCtx*)h;
  const double U_unit = 1.0;
  int L = c->maxlevel;
  int mech_it = 0, pf_it = 0;
  // the reference's own u_entire / phase_field at its thresholds, the tolerance drivers otherwise
  int mech_cy = mech_tol == 1e-6 ? ref_u_entire(h, mg_u, small_k, U_unit, t, &c->f_norm, &mech_it)
                                 : ref_u_entire_tol(h, mg_u, small_k, U_unit, t, &c->f_norm, &mech_it, mech_tol);
  if (t == 0) {
    if (ut0 <= 0.0) {
      c->Ue = ref_U_e(h, lc);
      c->Ut = c->Ue;
      c->delta_U = dU_factor * c->Ue;
    } else {
      c->Ue = ut0;
      c->Ut = ut0;
      c->delta_U = dU;
    }
    c->u_proportion = c->Ut / U_unit;
  }
  strain_history(&c->U, c->H->getLevel(L), c->u->getLevel(L), c->bulK->getLevel(L), c->G->getLevel(L),
                 c->gc->getLevel(L), c->M, L, lc, c->u_proportion);
  Voigt_all_level(*c->H, c->M);
  for (int l = L; l >= 0; l--) fd_h(&c->U, c->fd->getLevel(l), c->H->getLevel(l), l);
  int pf_cy = pf_tol == 1e-12 ? ref_phase_field(h, mg_d, lc, t, &c->fd_norm, &pf_it)
                              : ref_phase_field_tol(h, mg_d, lc, t, &c->fd_norm, &pf_it, pf_tol);
  double dd = delta_d_max(c->d->getLevel(L), *c->d_old);
  *c->d_old = c->d->getLevel(L);
  double FeW = externe_force_sum(c->fu->getLevel(L).getgrid(2), c->M) * voxel_size;
  double dmax = d_max(c->d->getLevel(L));
  double Ut_now = c->Ut;
  c->Ut = c->Ut + c->delta_U;
  c->u_proportion = c->Ut / U_unit;
  out[0] = Ut_now;
  out[1] = c->u_proportion * FeW;
  out[2] = dd;
  out[3] = dmax;
  out[4] = mech_cy;
  out[5] = pf_cy;
  out[6] = mech_it;
  out[7] = pf_it;
  return 0;
}

void ref_state(void* h, double* s6) {
  RefCtx* c = (RefCtx*)h;
  s6[0] = c->f_norm; s6[1] = c->fd_norm; s6[2] = c->Ue; s6[3] = c->Ut; s6[4] = c->delta_U;
  s6[5] = c->u_proportion;
}
void ref_set_state(void* h, const double* s6) {
  RefCtx* c = (RefCtx*)h;
  c->f_norm = s6[0]; c->fd_norm = s6[1]; c->Ue = s6[2]; c->Ut = s6[3]; c->delta_U = s6[4];
  c->u_proportion = s6[5];
}

/* Text the reference printed during the last captured call (residual history). */
const char* ref_last_output(void) { return g_last_out.c_str(); }

// write_vector_3D / read_vector_3D (write_read_history.cpp:18-86) of one grid; `path` ends in
// ".dat", so the reference uses it as given.
int ref_write_vector_3d(void* h, int field, int level, int comp, const char* path, int t) {
  griddouble* g = grid_of((RefCtx*)h, field, level, comp);
  if (!g) return -1;
  captured([&] { write_vector_3D(*g, std::string(path), 0, t); });
  return 0;
}
int ref_read_vector_3d(void* h, int field, int level, int comp, const char* path, int t) {
  griddouble* g = grid_of((RefCtx*)h, field, level, comp);
  if (!g) return -1;
  captured([&] { read_vector_3D(*g, std::string(path), 0, t); });
  return 0;
}

// write_total_de ("S"), write_total_u ("V", scaled by u_proportion) or write_total_H ("C") of
// vtk_output.cpp:420-469 for one rank, run in `workdir` (the reference writes below ./Output).
int ref_write_vtk(void* h, const char* option, int field, int level, const char* filename, const char* field_name,
                  int t, double u_proportion, const char* workdir) {
  RefCtx* c = (RefCtx*)h;
  char cwd[4096];
  if (!getcwd(cwd, sizeof cwd) || chdir(workdir) != 0) return -1;
  int rc = 0;
  const std::string opt(option);
  captured([&] {
    if (opt == "S") {
      griddouble* g = grid_of(c, field, level, 0);
      if (g) write_total_de(&c->U, *g, c->M, opt, filename, field_name, level, 0, 1, t);
      else rc = -1;
    } else if (opt == "V") {
      mgvecdouble* v = vector_field(c, field);
      if (v) write_total_u(&c->U, v->getLevel(level), c->M, level, 0, 1, filename, field_name, t, u_proportion);
      else rc = -1;
    } else if (opt == "C") {
      griddouble* g = grid_of(c, field, level, 0);
      if (g) write_total_H(&c->U, *g, c->M, opt, filename, field_name, level, 0, 1, t);
      else rc = -1;
    } else {
      rc = -1;
    }
  });
  if (chdir(cwd) != 0) return -1;
  return rc;
}

}  // extern "C"
