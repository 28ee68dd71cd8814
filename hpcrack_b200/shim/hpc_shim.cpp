// Drop-in replacements, with the reference's exact signatures, for the HPCrack functions on the
// fracture hot path.  Linked in place of the reference's translation units
//   mechanical_pcg.cpp, mechanical_multigrid.cpp, mechanical_displacement.cpp,
//   phase_field_pcg.cpp, phase_field_multigrid.cpp, phase_field.cpp,
//   strain_history.cpp, phase_field_max_search.cpp
// they move the work to the B200 library through its C ABI (include/hpcrack.h).  The caller's
// grid<T> / mg<T> / mgvec<T> storage stays the source of truth: every call uploads the fields it
// reads and downloads the fields it writes, so any mix of shimmed and reference functions keeps
// the reference's data flow.  (The device-resident loop in hpc_shim_loop.cpp avoids these copies.)
//
// One device context is created per Stack on first use.  MPI_Setting arguments are accepted and
// ignored: one rank, no halo.  Errors are thrown as std::runtime_error, as the reference does.
#include <cmath>
#include <map>
#include <stdexcept>
#include <string>

#include "mpi_struct.h"
#include "mgvec.h"
#include "mechanical_pcg.h"
#include "phase_field_pcg.h"
#include "mechanical_multigrid.h"
#include "phase_field_multigrid.h"
#include "mechanical_displacement.h"
#include "phase_field.h"
#include "strain_history.h"
#include "phase_field_max_search.h"
#include "mechanical_strain.h"
#include "hpcrack.h"
#include "hpc_shim.h"

namespace {

std::map<const Stack*, hpc_ctx*>& contexts() {
  static std::map<const Stack*, hpc_ctx*> m;
  return m;
}
hpc_ctx* g_current = nullptr;

void check(int rc, const char* what) {
  if (rc != HPC_OK) throw std::runtime_error(std::string(what) + ": " + hpc_last_error());
}

// Level sizes of a Stack built by initialize() for one rank (initialization.cpp:19-134).
hpc_geometry geometry_of(const Stack* U) {
  hpc_geometry g{};
  g.maxlevel = U->maxlevel;
  const Level* L0 = U->Ll;
  g.element_nb[0] = (int)L0->ii;
  g.element_nb[1] = (int)L0->jj;
  g.element_nb[2] = (int)L0->kk;
  g.x_start[0] = U->xa;
  g.x_start[1] = U->ya;
  g.x_start[2] = U->za;
  const double span[3] = {U->xb - U->xa, U->yb - U->ya, U->zb - U->za};
  for (int a = 0; a < 3; ++a)
    g.roi_start[a] = (int)std::lround(span[a] - g.element_nb[a] * std::pow(2.0, U->maxlevel));
  return g;
}

int level_of(const Stack* U, size_t n) {
  for (int l = 0; l <= U->maxlevel; ++l) {
    const Level* L = U->Ll + l;
    if ((size_t)L->nbcolox * L->nbcoloy * L->nbcoloz == n) return l;
  }
  throw std::runtime_error("grid size matches no level of the hierarchy");
}

template <class T>
T* data(grid<T>& g) { return &g[0]; }
template <class T>
const T* data(const grid<T>& g) { return &g[0]; }

void put(hpc_ctx* c, int field, int l, int comp, const griddouble& g) {
  check(hpc_upload(c, field, l, comp, data(g)), "hpc_upload");
}
void get(hpc_ctx* c, int field, int l, int comp, griddouble& g) {
  check(hpc_download(c, field, l, comp, data(g)), "hpc_download");
}
void putv(hpc_ctx* c, int field, int l, const gdvecdouble& v) {
  for (int di = 0; di < 3; ++di) put(c, field, l, di, v.getgrid(di));
}
void getv(hpc_ctx* c, int field, int l, gdvecdouble& v) {
  for (int di = 0; di < 3; ++di) get(c, field, l, di, v.getgrid(di));
}
void put_choice(hpc_ctx* c, int l, const gridshort& g) {
  check(hpc_upload_choice(c, l, reinterpret_cast<const int16_t*>(data(g))), "hpc_upload_choice");
}

hpc_mg mg_of(const MG& m) { return hpc_mg{m.nu0, m.nu1, m.nu2, m.gamma, m.ncy}; }

// Uploads the level-l inputs of the mechanical operator.
void put_mech_level(hpc_ctx* c, int l, const gridshort& choice, const griddouble& bulK, const griddouble& G,
                    const griddouble& d, const griddouble& Ke, const griddouble& Ge) {
  put_choice(c, l, choice);
  put(c, HPC_BULK, l, 0, bulK);
  put(c, HPC_G, l, 0, G);
  put(c, HPC_D, l, 0, d);
  put(c, HPC_KE, l, 0, Ke);
  put(c, HPC_GE, l, 0, Ge);
}

}  // namespace

hpc_ctx* hpc_shim_context(Stack* U) {
  auto& m = contexts();
  auto it = m.find(U);
  if (it != m.end()) return g_current = it->second;
  hpc_geometry g = geometry_of(U);
  hpc_ctx* c = nullptr;
  check(hpc_create(&c, &g, 0), "hpc_create");
  m[U] = c;
  return g_current = c;
}

void hpc_shim_release_all() {
  for (auto& kv : contexts()) hpc_destroy(kv.second);
  contexts().clear();
  g_current = nullptr;
}

// ------------------------------------------------------------------ mechanical_pcg.h
void Internal_Force(Stack* U, gdvecdouble& Fi, const gdvecdouble& u, const gridshort& MP_choice_d,
                    const griddouble& bulK, const griddouble& G, const griddouble& d, const griddouble& K_element,
                    const griddouble& G_element, const griddouble& DN, const grid2d& N, const double wg, const int l,
                    const double small_k) {
  (void)DN; (void)N; (void)wg;  // the library derives the shape tables of level l itself
  hpc_ctx* c = hpc_shim_context(U);
  put_mech_level(c, l, MP_choice_d, bulK, G, d, K_element, G_element);
  putv(c, HPC_U, l, u);
  check(hpc_internal_force(c, l, HPC_U, HPC_RU, small_k), "Internal_Force");
  getv(c, HPC_RU, l, Fi);
}

void PreM_u(Stack* U, gdvecdouble& preM, const gridshort& MP_choice_d, const griddouble& bulK, const griddouble& G,
            const griddouble& d, const griddouble& K_element, const griddouble& G_element, const griddouble& DN,
            const grid2d& N, const double wg, const int l, const double small_k) {
  (void)DN; (void)N; (void)wg;
  hpc_ctx* c = hpc_shim_context(U);
  put_mech_level(c, l, MP_choice_d, bulK, G, d, K_element, G_element);
  check(hpc_prem_u(c, l, HPC_RU, small_k), "PreM_u");
  // PreM_u accumulates into preM (mechanical_pcg.cpp:95-97); callers pass a zeroed grid
  gdvecdouble diag(3, preM.getgrid(0).axis());
  getv(c, HPC_RU, l, diag);
  for (int di = 0; di < 3; ++di) preM.getgrid(di) += diag.getgrid(di);
}

double Initial_residual_u(Stack* U, gdvecdouble& ru, const gdvecdouble& u, const gdvecdouble& fu,
                          const gridshort& MP_choice_d, const griddouble& bulK, const griddouble& G,
                          const griddouble& d, const griddouble& K_element, const griddouble& G_element,
                          MPI_Setting& M, const int l, const double small_k) {
  (void)M;
  hpc_ctx* c = hpc_shim_context(U);
  put_mech_level(c, l, MP_choice_d, bulK, G, d, K_element, G_element);
  putv(c, HPC_U, l, u);
  putv(c, HPC_FU, l, fu);
  double r = 0.0;
  check(hpc_initial_residual_u(c, l, small_k, &r), "Initial_residual_u");
  getv(c, HPC_RU, l, ru);
  return r;
}

void pcg_u(Stack* U, gdvecdouble& u, gdvecdouble& ru, gdvecdouble& fu, const gridshort& MP_choice_d,
           const griddouble& bulK, const griddouble& G, const griddouble& d, const griddouble& K_element,
           const griddouble& G_element, MPI_Setting& M, const int l, const double small_k, const double Ut,
           const int NB_relax, const int t, double& f_norm) {
  (void)M;
  hpc_ctx* c = hpc_shim_context(U);
  put_mech_level(c, l, MP_choice_d, bulK, G, d, K_element, G_element);
  putv(c, HPC_U, l, u);
  putv(c, HPC_FU, l, fu);
  check(hpc_pcg_u(c, l, small_k, Ut, NB_relax, t, &f_norm), "pcg_u");
  getv(c, HPC_U, l, u);
  getv(c, HPC_RU, l, ru);
  getv(c, HPC_FU, l, fu);
}

// ------------------------------------------------------------------ mechanical_multigrid.h
void cycle_u(Stack* U, mgvecdouble& u, mgvecdouble& ru, mgvecdouble& fu, mgvecdouble& uold,
             const mgshort& MP_choice_d, const mgdouble& bulK, const mgdouble& G, const mgdouble& d,
             const mgdouble& K_element, const mgdouble& G_element, int l, const MG& mgp_u, MPI_Setting& M,
             const int myid, const int nbprocs, const double small_k, const double Ut, const int t, double& f_norm) {
  (void)M; (void)myid; (void)nbprocs;
  hpc_ctx* c = hpc_shim_context(U);
  for (int k = 0; k <= l; ++k) {
    put_mech_level(c, k, MP_choice_d.getLevel(k), bulK.getLevel(k), G.getLevel(k), d.getLevel(k),
                   K_element.getLevel(k), G_element.getLevel(k));
    putv(c, HPC_U, k, u.getLevel(k));
    putv(c, HPC_FU, k, fu.getLevel(k));
  }
  const hpc_mg mg = mg_of(mgp_u);
  check(hpc_cycle_u(c, l, &mg, small_k, Ut, t, &f_norm), "cycle_u");
  for (int k = 0; k <= l; ++k) {
    getv(c, HPC_U, k, u.getLevel(k));
    getv(c, HPC_RU, k, ru.getLevel(k));
    getv(c, HPC_FU, k, fu.getLevel(k));
    if (k < l && k < uold.nbl()) getv(c, HPC_UOLD, k, uold.getLevel(k));
  }
}

// ------------------------------------------------------------------ mechanical_displacement.h
void u_entire(Stack* U, mgvecdouble& u, mgvecdouble& fu, const mgdouble& bulK, const mgdouble& G, const mgdouble& d,
              MPI_Setting& M, const MG& mgp_u, const int myid, const int nbprocs, const double small_k,
              const double Ut, const int t, double& f_norm) {
  (void)M; (void)myid; (void)nbprocs;
  hpc_ctx* c = hpc_shim_context(U);
  const int L = U->maxlevel;
  for (int k = 0; k <= L; ++k) {
    put(c, HPC_BULK, k, 0, bulK.getLevel(k));
    put(c, HPC_G, k, 0, G.getLevel(k));
    put(c, HPC_D, k, 0, d.getLevel(k));
  }
  putv(c, HPC_U, L, u.getLevel(L));
  putv(c, HPC_FU, L, fu.getLevel(L));
  const hpc_mg mg = mg_of(mgp_u);
  int cycles = 0, iters = 0;
  check(hpc_u_entire(c, &mg, small_k, Ut, t, &f_norm, 1e-6, &cycles, &iters), "u_entire");
  for (int k = 0; k <= L; ++k) getv(c, HPC_U, k, u.getLevel(k));
  getv(c, HPC_FU, L, fu.getLevel(L));
}

// ------------------------------------------------------------------ phase_field_pcg.h
void Fld(grid<double>& Fi, const grid<double>& d, const grid<double>& H, const grid<double>& gc,
         const grid<double>& DN, const grid2d& N, const double lc, const double wg) {
  (void)DN; (void)N; (void)wg;
  if (!g_current) throw std::runtime_error("Fld: no hierarchy context yet");
  // the level is identified by the grid size within the current hierarchy
  int n3[3];
  int l = -1;
  for (int k = 0; k < 16; ++k) {
    if (hpc_level_dims(g_current, k, n3, nullptr) != HPC_OK) break;
    if ((size_t)n3[0] * n3[1] * n3[2] == const_cast<grid<double>&>(d).size()) l = k;
  }
  if (l < 0) throw std::runtime_error("Fld: grid size matches no level");
  put(g_current, HPC_R, l, 0, d);
  put(g_current, HPC_H, l, 0, H);
  put(g_current, HPC_GC, l, 0, gc);
  check(hpc_fld(g_current, l, HPC_R, HPC_FD, lc), "Fld");
  get(g_current, HPC_FD, l, 0, Fi);
}

void Precondition_M(grid<double>& Md, const grid<double>& H, const grid<double>& gc, const grid<double>& DN,
                    grid2d& N, const double lc, const double wg) {
  (void)DN; (void)N; (void)wg;
  if (!g_current) throw std::runtime_error("Precondition_M: no hierarchy context yet");
  int n3[3];
  int l = -1;
  for (int k = 0; k < 16; ++k) {
    if (hpc_level_dims(g_current, k, n3, nullptr) != HPC_OK) break;
    if ((size_t)n3[0] * n3[1] * n3[2] == Md.size()) l = k;
  }
  if (l < 0) throw std::runtime_error("Precondition_M: grid size matches no level");
  put(g_current, HPC_H, l, 0, H);
  put(g_current, HPC_GC, l, 0, gc);
  check(hpc_precondition_m(g_current, l, HPC_R, lc), "Precondition_M");
  get(g_current, HPC_R, l, 0, Md);
}

double initial_residual(Stack* U, grid<double>& R, grid<double>& d, const grid<double>& fd, const grid<double>& H,
                        const grid<double>& gc, const int l, const double lc, const MPI_Setting& M) {
  (void)M;
  hpc_ctx* c = hpc_shim_context(U);
  put(c, HPC_D, l, 0, d);
  put(c, HPC_FD, l, 0, fd);
  put(c, HPC_H, l, 0, H);
  put(c, HPC_GC, l, 0, gc);
  double r = 0.0;
  check(hpc_initial_residual_d(c, l, lc, &r), "initial_residual");
  get(c, HPC_R, l, 0, R);
  return r;
}

void pcg_d(Stack* U, grid<double>& d, grid<double>& fd, grid<double>& R, const grid<double>& H,
           const grid<double>& gc, MPI_Setting& M, const int l, const double lc, const int NB_relax, const int t,
           double& fd_norm) {
  (void)M;
  hpc_ctx* c = hpc_shim_context(U);
  put(c, HPC_D, l, 0, d);
  put(c, HPC_FD, l, 0, fd);
  put(c, HPC_H, l, 0, H);
  put(c, HPC_GC, l, 0, gc);
  check(hpc_pcg_d(c, l, lc, NB_relax, t, &fd_norm), "pcg_d");
  get(c, HPC_D, l, 0, d);
  get(c, HPC_R, l, 0, R);
}

// ------------------------------------------------------------------ phase_field_multigrid.h / phase_field.h
void cycle_d(Stack* U, mg<double>& d, mg<double>& fd, mg<double>& dold, const mg<double>& H, const mg<double>& gc,
             mg<double>& r, int l, const double lc, const MG& mgp_d, MPI_Setting& M, const int myid,
             const int nbprocs, const int t, double& fd_norm) {
  (void)M; (void)myid; (void)nbprocs;
  hpc_ctx* c = hpc_shim_context(U);
  for (int k = 0; k <= l; ++k) {
    put(c, HPC_D, k, 0, d.getLevel(k));
    put(c, HPC_FD, k, 0, fd.getLevel(k));
    put(c, HPC_H, k, 0, H.getLevel(k));
    put(c, HPC_GC, k, 0, gc.getLevel(k));
  }
  const hpc_mg mg = mg_of(mgp_d);
  check(hpc_cycle_d(c, l, &mg, lc, t, &fd_norm), "cycle_d");
  for (int k = 0; k <= l; ++k) {
    get(c, HPC_D, k, 0, d.getLevel(k));
    get(c, HPC_FD, k, 0, fd.getLevel(k));
    get(c, HPC_R, k, 0, r.getLevel(k));
    if (k < l && k < dold.nbl()) get(c, HPC_DOLD, k, 0, dold.getLevel(k));
  }
}

void phase_field(Stack* U, mg<double>& d, mg<double>& fd, const mg<double>& H, const mg<double>& gc,
                 MPI_Setting& M, double lc, const MG& mgp_d, int myid, int nbprocs, int t, double& fd_norm) {
  (void)M; (void)myid; (void)nbprocs;
  hpc_ctx* c = hpc_shim_context(U);
  const int L = U->maxlevel;
  for (int k = 0; k <= L; ++k) {
    put(c, HPC_D, k, 0, d.getLevel(k));
    put(c, HPC_FD, k, 0, fd.getLevel(k));
    put(c, HPC_H, k, 0, H.getLevel(k));
    put(c, HPC_GC, k, 0, gc.getLevel(k));
  }
  const hpc_mg mg = mg_of(mgp_d);
  int cycles = 0, iters = 0;
  check(hpc_phase_field(c, &mg, lc, t, &fd_norm, 1e-12, &cycles, &iters), "phase_field");
  for (int k = 0; k <= L; ++k) {
    get(c, HPC_D, k, 0, d.getLevel(k));
    get(c, HPC_FD, k, 0, fd.getLevel(k));
  }
}

// ------------------------------------------------------------------ strain_history.h
// Per-Gauss-point helpers stay host functions (material_selection.cpp calls them); they restate
// strain_history.cpp:134-159 in this library's own code.
double Phi_c(const double gc_g, const double lc) { return 0.5 * gc_g / lc; }

double W(const grid2d& sigma, const grid2d& epsilon) {
  double w = 0.;
  for (int c = 0; c < 3; c++)
    for (int m = 0; m < 3; m++) w += 0.5 * sigma(c, m) * epsilon(c, m);
  return w;
}

double Phi_positive(const double K_g, const double G_g, const grid2d& epsilon) {
  const double tr = trace_epsilon(epsilon);
  const double dev = epsilon_dev(epsilon);
  return tr >= 0 ? 0.5 * K_g * tr * tr + G_g * dev : G_g * dev;
}

double Phi_negative(const double K_g, const grid2d& epsilon) {
  const double tr = trace_epsilon(epsilon);
  return tr >= 0 ? 0.0 : 0.5 * K_g * tr * tr;
}

void initial_crack(Stack* U, griddouble& H, const MPI_Setting& M, const double H_crack, const int l) {
  (void)M;
  hpc_ctx* c = hpc_shim_context(U);
  put(c, HPC_H, l, 0, H);
  check(hpc_initial_crack(c, H_crack, l), "initial_crack");
  get(c, HPC_H, l, 0, H);
}

double U_e(Stack* U, const gdvecdouble& u, const griddouble& bulK, const griddouble& G, const griddouble& gc,
           const int l, const double lc, const MPI_Setting& M) {
  (void)M;
  hpc_ctx* c = hpc_shim_context(U);
  if (l != U->maxlevel) throw std::runtime_error("U_e: the library evaluates it on the finest level");
  putv(c, HPC_U, l, u);
  put(c, HPC_BULK, l, 0, bulK);
  put(c, HPC_G, l, 0, G);
  put(c, HPC_GC, l, 0, gc);
  double ue = 0.0;
  check(hpc_U_e(c, lc, &ue), "U_e");
  return ue;
}

void strain_history(Stack* U, griddouble& H, const gdvecdouble& u, const griddouble& bulK, const griddouble& G,
                    const griddouble& gc, const MPI_Setting& M, const int l, const double lc,
                    const double u_proportion) {
  (void)M;
  hpc_ctx* c = hpc_shim_context(U);
  if (l != U->maxlevel) throw std::runtime_error("strain_history: the library evaluates it on the finest level");
  put(c, HPC_H, l, 0, H);
  putv(c, HPC_U, l, u);
  put(c, HPC_BULK, l, 0, bulK);
  put(c, HPC_G, l, 0, G);
  put(c, HPC_GC, l, 0, gc);
  check(hpc_strain_history(c, lc, u_proportion), "strain_history");
  get(c, HPC_H, l, 0, H);
}

// ------------------------------------------------------------------ phase_field_max_search.h
static int finest_of_size(size_t n) {
  if (!g_current) throw std::runtime_error("d_max: no hierarchy context yet");
  int n3[3];
  for (int k = 15; k >= 0; --k) {
    if (hpc_level_dims(g_current, k, n3, nullptr) != HPC_OK) continue;
    if ((size_t)n3[0] * n3[1] * n3[2] == n) return k;
    break;
  }
  throw std::runtime_error("d_max: the library evaluates it on the finest level");
}

double delta_d_max(const grid<double>& d, const grid<double>& d_old) {
  const int l = finest_of_size(const_cast<grid<double>&>(d).size());
  put(g_current, HPC_D, l, 0, d);
  put(g_current, HPC_DOLDF, l, 0, d_old);
  double v = 0.0;
  check(hpc_delta_d_max(g_current, &v), "delta_d_max");
  return v;
}

double d_max(const grid<double>& d) {
  const int l = finest_of_size(const_cast<grid<double>&>(d).size());
  put(g_current, HPC_D, l, 0, d);
  double v = 0.0;
  check(hpc_d_max(g_current, &v), "d_max");
  return v;
}
