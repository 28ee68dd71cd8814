/*
 * hpc_oracle.h - plain-C restatement of the HPCrack hot path.
 *
 * TEST INFRASTRUCTURE.  This is the CPU oracle that the CUDA library is checked
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it.  Its parity with the reference itself is pinned by golden
 * vectors produced by the reference compiled from its own sources
 * (tests/golden/make_golden.py over oracle/_ref/libhpcref.so).
 *
 * Layout (same as the reference, include/grid.h:83-91): a level is a dense
 * nx*ny*nz array, x fastest; element (i,j,k) data live at node (i,j,k) of a
 * node-sized array.  Vector fields are three such arrays back to back
 * (component 0, 1, 2).  Level 0 is the coarsest (include/mg.h:54-65).
 */
#ifndef HPC_ORACLE_H
#define HPC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXL 16

typedef struct {
  int nx, ny, nz;
  double hx, hy, hz;
} orc_lvl;

typedef struct {
  int maxlevel;
  int enb[3];
  int roi[3];
  double x0[3];
  double box[6]; /* xa xb ya yb za zb */
  orc_lvl lv[ORC_MAXL];
} orc_geom;

/* Field ids shared with oracle/ref_harness.cpp. */
enum {
  ORC_BULK = 0, ORC_G = 1, ORC_GC = 2, ORC_D = 3, ORC_H = 4, ORC_FD = 5, ORC_KE = 6, ORC_GE = 7,
  ORC_R = 8, ORC_DOLD = 9, ORC_DOLDF = 10,
  ORC_U = 16, ORC_FU = 17, ORC_RU = 18, ORC_UOLD = 19,
  ORC_CHOICE = 32
};

typedef struct orc_state orc_state;

/* geometry (initialization.cpp:19-134 with input_setting, image_input.cpp:21-27) */
void orc_geom_init(orc_geom* g, int maxlevel, const int* enb, const double* x0, const int* roi);

/* ---- single-level kernels on raw arrays ---- */
int orc_internal_force(const orc_lvl* L, int finest, const double* u, const short* choice,
                       const double* bulK, const double* G, const double* d, const double* Ke,
                       const double* Ge, double small_k, double* Fi);
int orc_prem_u(const orc_lvl* L, int finest, const short* choice, const double* bulK, const double* G,
               const double* d, const double* Ke, const double* Ge, double small_k, double* preM);
void orc_fld(const orc_lvl* L, const double* x, const double* H, const double* gc, double lc, double* Fi);
void orc_precondition_m(const orc_lvl* L, const double* H, const double* gc, double lc, double* Md);
void orc_injection(const orc_lvl* Lc, const orc_lvl* Lf, const double* uf, double* uc);
void orc_restrict(const orc_lvl* Lc, const orc_lvl* Lf, const double* rf, const double* Fic, double* fc);
void orc_prolong(const orc_lvl* Lc, const orc_lvl* Lf, const double* uc, const double* ucold, double* uf);

/* ---- hierarchy state mirroring the reference's mg / mgvec containers ---- */
orc_state* orc_state_create(int maxlevel, const int* enb, const double* x0, const int* roi);
void orc_state_destroy(orc_state* s);
const orc_geom* orc_state_geom(const orc_state* s);
int orc_set(orc_state* s, int field, int level, int comp, const double* src);
int orc_get(orc_state* s, int field, int level, int comp, double* dst);
int orc_set_choice(orc_state* s, int level, const short* src);
int orc_get_choice(orc_state* s, int level, short* dst);
void orc_set_choice_quirk(orc_state* s, int reproduce);
void orc_state_scalars(orc_state* s, double* s6);
void orc_set_state_scalars(orc_state* s, const double* s6);

int orc_st_internal_force(orc_state* s, int level, int src, int dst, double small_k);
int orc_st_prem_u(orc_state* s, int level, int dst, double small_k);
int orc_st_fld(orc_state* s, int level, int src, int dst, double lc);
int orc_st_precondition_m(orc_state* s, int level, int dst, double lc);
int orc_dirichlet_bd(orc_state* s, int level, int field, double Ut);
int orc_dirichlet_force(orc_state* s, int level, int f_field, int fi_field);
int orc_dirichlet_residual(orc_state* s, int level, int field);

double orc_initial_residual_u(orc_state* s, int level, double small_k);
int orc_pcg_u(orc_state* s, int level, double small_k, double Ut, int nb_relax, int t, double* f_norm);
double orc_initial_residual_d(orc_state* s, int level, double lc);
int orc_pcg_d(orc_state* s, int level, double lc, int nb_relax, int t, double* fd_norm);
int orc_cycle_u(orc_state* s, int level, const int* mg5, double small_k, double Ut, int t, double* f_norm);
int orc_cycle_d(orc_state* s, int level, const int* mg5, double lc, int t, double* fd_norm);
int orc_u_entire(orc_state* s, const int* mg5, double small_k, double Ut, int t, double* f_norm,
                 int* iters, double mech_tol);
int orc_phase_field(orc_state* s, const int* mg5, double lc, int t, double* fd_norm, int* iters,
                    double pf_tol);

void orc_mp_choice(orc_state* s);
void orc_mp_all_element(orc_state* s, double small_k);
int orc_vr_all_level(orc_state* s, int field);
int orc_voigt_all_level(orc_state* s, int field);
int orc_coarse_vr(orc_state* s, int field);
void orc_strain_history(orc_state* s, double lc, double u_proportion);
void orc_fd_h(orc_state* s, int level);
double orc_delta_d_max(orc_state* s);
double orc_d_max(orc_state* s);
double orc_U_e(orc_state* s, double lc);
void orc_externe_force_nodal(orc_state* s, double Ut, double small_k);
double orc_externe_force_sum(orc_state* s);
void orc_initial_crack(orc_state* s, double H_crack, int level);
int orc_solution_injection(orc_state* s, int field, int comp, int lf);
int orc_coarsen_f_standard(orc_state* s, int fc_field, int rf_field, int fic_field, int comp, int lf);
int orc_refine_standard(orc_state* s, int uf_field, int uc_field, int ucold_field, int comp, int lf);

/* image + CSV material table -> finest bulK, G, gc (image_input.cpp:120-142), then coarse_VR. */
int orc_image_material(orc_state* s, const unsigned char* image, const int* voxel_n, int ngray,
                       const int* gray, const double* E, const double* nu, const double* gcv,
                       double voxel_size);

int orc_step(orc_state* s, int t, const int* mg_u, const int* mg_d, double small_k, double lc,
             double voxel_size, double ut0, double dU, double dU_factor, double mech_tol, double pf_tol,
             double* out);

#ifdef __cplusplus
}
#endif
#endif
