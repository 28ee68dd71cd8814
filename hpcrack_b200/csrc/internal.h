// Internal declarations of the B200 HPCrack library: context, level descriptors and kernel
// launchers.  Host code is C++17; device code is CUDA for sm_100a.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>

#include "../../include/hpcrack.h"

namespace hpc {

constexpr int kMaxLevels = 16;
constexpr int kPitchAlign = 4;  // x pitch rounded to 4 doubles (32 B): 16-byte aligned rows

// Geometry of one level as the kernels see it.  Arrays are x-fastest with an x pitch `px` >= nx;
// padding slots are kept at zero in every vector and diagonal, so flat vector kernels may run over
// the padded range.
struct LevelGeo {
  int nx, ny, nz, px;
  long long plane;  // px * ny
  long long n;      // px * ny * nz (padded slots)
  double hx, hy, hz, wg;
  // Dirichlet node sets, selected by floating-point coordinate equality exactly as
  // boundary_conditions.cpp:20-68 does; they are separable per axis:
  //   bx[i] bit0: x == (xa+xb)/2   bit1: x == xb
  //   by[j] bit0: y == ya          bit1: y == (ya+yb)/2
  //   bz[k] bit0: z == za          bit1: z == zb
  const uint8_t* bx;
  const uint8_t* by;
  const uint8_t* bz;
  // z-slab decomposition (one specimen split along z over ranks, initialization.cpp:19-134): the
  // global z index of local plane 0 (get_coordinate, boundary_conditions.cpp:13-18), the planes
  // this rank owns [oz0, oz1) (realdomain.h:17-40; the others are ghost copies of a neighbour's
  // planes), and on a coarse level the shift of its fine level: coarse plane kc sits on fine
  // local plane 2 kc + zsh (0, or -1 on every rank but the first).  One rank: 0, [0, nz), 0.
  int zb, oz0, oz1, zsh;
};

struct LevelFields {
  double *bulK, *G, *gc, *d, *H, *fd, *Ke, *Ge, *R, *dold;
  double *u, *fu, *ru, *uold;  // 3n each; component c at +c*n
  int8_t* choice;
  // work arrays
  double *preMu, *p, *w, *tmp3;  // 3n; preMu holds the inverse diagonal while a solve runs
  double *preMd, *pd, *wd, *tmp1;  // n;  preMd likewise
  uint8_t* bc_host_copy;           // host copies of the axis flags (nx+ny+nz bytes)
  double* gpm;  // finest level: Gauss-point moduli of the running mechanical solve, 16n (first use)
};

// Single-precision mirror of one level for the V-cycle of the precision form (hpc_step with
// mech_solver HPC_MECH_MIXED): vectors 3n floats, material n floats, allocated on first use.
struct LevelF32 {
  float *u, *fu, *ru, *uold, *p, *w, *invM;  // 3n each; invM: inverse diagonal of K
  float *K, *G, *d;                           // finest level: nodal moduli and phase field
  float *Ke, *Ge;                             // coarse levels: element moduli
  float* gpm;                                 // finest level: Gauss-point moduli, 16n
};

// Device scalar pool layout (doubles).
enum Scalar : int {
  S_FNORM = 0,    // f_norm of the mechanical solve (pcg_u at t == 0, finest)
  S_FDNORM = 1,   // fd_norm (rewritten by every pcg_d)
  S_RNORM = 2,    // last squared residual norm
  S_RES0 = 3,     // generic reduction results
  S_RES1 = 4,
  S_RES2 = 5,
  S_ERR = 6,      // set to 1 by a kernel whose bounded wait ran out (tensor-core apply)
  S_LCOUNT = 7,   // device-driven solve loops (batched steps): cycles run,
  S_LREL = 8,     //   the convergence ratio the loop tests,
  S_LTRUE = 9,    //   true-residual recomputations of the flexible PCG
  S_PCG = 16,     // pcg scratch: rz[-1..kMaxRelax], pw[0..kMaxRelax), rn[0..kMaxRelax)
};
constexpr int kMaxRelax = 4096;
constexpr int S_ZEROS = S_PCG + 3 * (kMaxRelax + 2);  // zero-diagonal counts, one slot per level
// flexible-PCG outer solve: per iteration k, delta = (z_k, r_k), gamma = (z_k, r_{k-1}), (p_k, w_k),
// |r_{k+1}|^2 and (r, M^-1 r) (unused)
constexpr int S_FCG = S_ZEROS + 16;
constexpr int kScalarPool = S_FCG + 5 * (kMaxRelax + 2);
inline int slot_rz(int it) { return S_PCG + 1 + it; }  // it >= -1
inline int slot_pw(int it) { return S_PCG + (kMaxRelax + 2) + it; }
inline int slot_rn(int it) { return S_PCG + 2 * (kMaxRelax + 2) + it; }
// Flexible-PCG scalars of iteration k >= -1: two sets by the parity of k (iteration k reads its own
// and the previous iteration's), so that every iteration of one parity launches the same arguments
// and can be replayed from one CUDA graph.
inline int slot_fdelta(int k) { return S_FCG + (k & 1); }
inline int slot_fgamma(int k) { return S_FCG + 2 + (k & 1); }
inline int slot_fpw(int k) { return S_FCG + 4 + (k & 1); }
inline int slot_frn(int k) { return S_FCG + 6 + (k & 1); }
inline int slot_fdummy(int k) { return S_FCG + 8 + (k & 1); }

}  // namespace hpc

struct hpc_ctx {
  unsigned long long uid;  // unique per context of the process (keys of the batched graphs)
  hpc_geometry geo;
  int maxlevel;
  double box[6];  // xa xb ya yb za zb
  hpc::LevelGeo L[hpc::kMaxLevels];
  hpc::LevelFields F[hpc::kMaxLevels];
  hpc::LevelF32 F32[hpc::kMaxLevels];  // precision form (null until first used)
  double* d_old;  // finest d of the previous increment
  cudaStream_t stream;
  int device;
  double* scal;          // device scalar pool
  double* hscal;         // pinned host staging for scalar reads
  double* stage;         // dense finest-size device buffer for uploads (first use)
  double* partials;      // per-block reduction partials
  unsigned int* counter; // last-block-done counter
  size_t partials_cap;   // doubles
  void* bc_dev_base;     // one allocation for all axis flags
  long long launches;
  int choice_quirk;
  // CUDA graphs of the coarse part of a V-cycle (everything below the finest level), cached with
  // the parameters they were captured for
  struct CoarseGraph {
    cudaGraphExec_t exec;
    long long kernels;
    int valid;
    hpc_mg mg;
    double a, b;  // small_k, Ut (mechanical) or lc (phase field)
    int flags;    // kernel choices baked into the launches
  } gmech, gpf, g32;  // g32: FP32 coarse part of the mixed-precision preconditioner
  CoarseGraph gfcg[3];  // precision form: one whole flexible-PCG iteration (k = 0, odd k, even k >= 2)
  int use_graphs;
  int autotune;  // measure strip shapes on first use (hpc_set_autotune)
  int tc_apply;        // precision form: element contraction on the tensor cores (hpc_set_tensor_apply)
  int fused_coarsest;  // coarse-level pcg_u in one block when the level fits (hpc_set_fused_coarsest)
  int gpm_active;      // finest applies read F[maxlevel].gpm (set while a mechanical solve runs)
  int tma_stage;       // finest applies stage rows with tensor copies (hpc_set_tma_staging)
  // z-slab rank of a specimen split over ranks (hpc_create_slab); null for a whole specimen.  A
  // reduction launched on a slab context is combined over the ranks right after its launch
  // (slab_after_launch): the launcher's make_red records its slots here.
  struct SlabState* slab;
  int red_slot[3], red_op, red_pending;
  // per-class launch timing (hpc_kernel_timing)
  int timing_class;
  cudaEvent_t* tev;  // 2 * tev_cap events: start/stop pairs
  int tev_cap, tev_used;
  double f_norm, fd_norm, Ue, Ut, dU, uprop;  // staggered-loop state (crack_propagation.cpp:32-39)
  // checkpoint (hpc_checkpoint_*): a dense device snapshot of the finest u, v, w, H, d, d_old, copied
  // to pinned host memory on a copy stream while the compute stream goes on
  struct Checkpoint {
    double* dev;   // 6 * nx*ny*nz doubles
    double* host;  // pinned, same size
    cudaStream_t stream;
    cudaEvent_t snap, done;
    int t, pending, valid;
    double state[6];
  } ck;
  // flexible-PCG outer solve of the precision form (hpc_u_entire_fcg): finest-level 3n vectors,
  // allocated on first use
  struct Fcg {
    double *x, *r, *rp, *f, *p;  // iterate, residual, previous residual, right-hand side (fu saved), direction
  } fcg;
  // VTK output (hpc_vtk_write): base64 characters of one field on the device and in pinned host
  // memory, a copy stream, and the host thread writing the files (allocated on first use)
  struct Vtk {
    char* dev;
    char* host;
    size_t cap;
    cudaStream_t stream;
    cudaEvent_t packed, copied;
    void* job;
  } vtk;
};

namespace hpc {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
int cuda_fail(cudaError_t e, const char* where);
#define HPC_CUDA(call)                                            \
  do {                                                            \
    cudaError_t _e = (call);                                      \
    if (_e != cudaSuccess) return ::hpc::cuda_fail(_e, #call);    \
  } while (0)
#define HPC_CHECK_LAUNCH(ctx)                                               \
  do {                                                                      \
    (ctx)->launches++;                                                      \
    cudaError_t _e = cudaGetLastError();                                    \
    if (_e != cudaSuccess) return ::hpc::cuda_fail(_e, "kernel launch");    \
    if ((ctx)->slab) {                                                      \
      const int _r = ::hpc::slab_after_launch(ctx);                         \
      if (_r) return _r;                                                    \
    }                                                                       \
  } while (0)
// Ghost planes of `ncomp` components (stride L[level].n elements of `elem` bytes) of a slab
// context refreshed from the neighbouring ranks (SendRecv, mpi_communications.h:24-47, in z);
// nothing for a whole specimen.
#define HPC_SLAB_HALO(ctx, level, ptr, ncomp, elem)                         \
  do {                                                                      \
    if ((ctx)->slab) {                                                      \
      const int _r = ::hpc::slab_halo(ctx, level, (void*)(ptr), ncomp, elem); \
      if (_r) return _r;                                                    \
    }                                                                       \
  } while (0)

// z-slab transport (slab.cu): the reduction recorded by make_red combined over the ranks (sum, max
// or min in rank order, the same on every rank), and the ghost-plane exchange.
int slab_after_launch(hpc_ctx* c);
int slab_halo(hpc_ctx* c, int level, void* v, int ncomp, int elem_bytes);
// Per-level z extents of rank r of nr (initialization.cpp:19-134, boundary_conditions.cpp:13-18,
// realdomain.h:17-40): local planes, global index of local plane 0, owned planes [lo, hi).
struct SlabLevel {
  int nz, zb, lo, hi;
};
bool slab_levels(const hpc_geometry& g, int nr, int r, SlabLevel* out);
int slab_attach(hpc_ctx* c, int nr, int r);  // a new context becomes rank r of nr
void slab_release(hpc_ctx* c);
// The coarsest level's pcg_u of a slab of several ranks, solved redundantly: every rank gathers the
// whole coarsest level (its owned planes from every rank) and runs the one-block solver on it, then
// keeps its own planes.  One exchange per visit instead of three collective steps per iteration.
// 0: the context holds the whole coarsest level (no split, or one rank); 1: a split whose whole
// coarsest level fits the one-block solver (slab_coarsest); 2: a split whose does not (per-iteration
// kernels with their collective steps).
int slab_coarsest_mode(hpc_ctx* c);
int slab_coarsest(hpc_ctx* c, double Ut, int nb);

// Launch timing: bracket a launch of class `cls` with events when that class is being timed.
void timing_begin(hpc_ctx* c, int cls);
void timing_end(hpc_ctx* c, int cls);

// ---------------------------------------------------------------- field access
double* scalar_field(hpc_ctx* c, int field, int level);  // nullptr if not a scalar field
double* vector_field(hpc_ctx* c, int field, int level);  // nullptr if not a vector field
int read_scalars(hpc_ctx* c, int first, int count, double* out);  // sync + D2H of scalar slots
int write_scalar(hpc_ctx* c, int slot, double v);
// Waits for a VTK write in flight and frees the VTK buffers (vtk_output.cu); returns that write's status.
int vtk_release(hpc_ctx* c);

// ---------------------------------------------------------------- kernel launchers
// Element operators (element_kernels.cu).  `src` is a 3n (mech) or n (pf) vector on level L.
enum MechEpi { EPI_PLAIN = 0, EPI_RESIDUAL = 1, EPI_PCG = 2, EPI_FAS = 3, EPI_REACTION = 4 };

struct MechCall {
  int level;
  bool finest;
  int epi;
  const double* src;  // u (PLAIN / RESIDUAL / FAS / REACTION) or p (PCG)
  double* out;        // Fi (PLAIN), r (RESIDUAL), w (PCG), fc (FAS), fu (REACTION: BC slots only)
  double small_k;
  // RESIDUAL: r = fu - K u, zero at Dirichlet nodes; optionally fu[bc] = (K u)[bc] and f_norm.
  double* fu;
  bool set_fnorm;     // t == 0 on the finest level (mechanical_pcg.cpp:252-258)
  const double* invM; // RESIDUAL: inverse diagonal for rz = sum r^2 invM (null: no rz)
  // FAS: fc = K_c u_c + full-weighting(rf)
  const double* rf;
  int fine_level;
  // reduction destinations (scalar slots, -1 = none)
  int s_out0, s_out1, s_out2;
};
int launch_mech(hpc_ctx* c, const MechCall& m);
int launch_mech_diag(hpc_ctx* c, int level, bool finest, double small_k, double* out);
// Gauss-point moduli of the finest level into F[maxlevel].gpm (from bulK, G, d and the regimes)
int launch_gp_material(hpc_ctx* c, double small_k);

// Single-precision operator on the FP32 mirror of a level (EPI_PLAIN, EPI_RESIDUAL, EPI_PCG, EPI_FAS);
// the residual zeroes Dirichlet rows and sums (r, M^-1 r) into s_out1 and |r|^2 into s_out2 in FP64.
struct MechCall32 {
  int level;
  bool finest;
  int epi;
  const float* src;
  float* out;
  double small_k;
  float* fu;          // RESIDUAL: right-hand side
  const float* invM;  // RESIDUAL: inverse diagonal for (r, M^-1 r)
  const float* rf;    // FAS: fine residual
  int fine_level;
  int s_out0, s_out1, s_out2;
};
int launch_mech_f32(hpc_ctx* c, const MechCall32& m);
// FP32 mirror: u += alpha p, r -= alpha w on F32[level] (Dirichlet rows zero), alpha = scal[s_num]/scal[s_den]
int launch_mech_update_f32(hpc_ctx* c, int level, int s_num, int s_den, int s_rz_next, int s_rn);
// FP32 mirror: p = r M^-1 + beta p (beta from scal, 0 if first)
int launch_dir_update_f32(hpc_ctx* c, int level, bool first, int s_rz, int s_rz_prev);
int launch_bc_zero_f32(hpc_ctx* c, int level, float* v);  // zero the Dirichlet rows of a 3n vector
// FP32 mirror: r = f (Dirichlet rows zero) and (r, M^-1 r) for a correction whose unknown is zero
int launch_residual_zero_f32(hpc_ctx* c, int level, int s_rz);
int launch_inject_u_f32(hpc_ctx* c, int lf);             // u_c = u_f(2i), Dirichlet rows 0, uold_c = u_c
int launch_prolong_f32(hpc_ctx* c, int lf);              // u_f += P(u_c - uold_c), Dirichlet rows 0
int launch_to_f32(hpc_ctx* c, const double* src, float* dst, long long n);
int launch_to_f64(hpc_ctx* c, const float* src, double* dst, long long n);
int launch_unpack(hpc_ctx* c, int level, const double* dense, double* dst);

struct PfCall {
  int level;
  int epi;  // EPI_PLAIN, EPI_RESIDUAL, EPI_PCG, EPI_FAS
  const double* src;
  double* out;
  double lc;
  const double* fd;     // RESIDUAL: R = fd - A d
  const double* invM;   // RESIDUAL: inverse diagonal for rz (null: no rz)
  const double* rf;
  int fine_level;
  int s_out0, s_out1, s_out2;
};
int launch_pf(hpc_ctx* c, const PfCall& p);
int launch_pf_diag(hpc_ctx* c, int level, double lc, double* out);

// Vector kernels (vector_kernels.cu).
// Mechanical CG update: alpha = scal[s_rz]/scal[s_pw]; u += alpha p; r -= alpha w; r = 0 on Dirichlet
// nodes; scal[s_rz_next] = sum r^2/preM; scal[s_rn] = sum r^2.
int launch_mech_update(hpc_ctx* c, int level, const double* p, int s_rz, int s_pw, int s_rz_next, int s_rn);
// Same on explicit arrays: x += alpha p, r -= alpha w (Dirichlet rows zero), alpha = scal[s_num]/scal[s_den].
int launch_mech_update_on(hpc_ctx* c, int level, double* x, double* r, const double* p, const double* w,
                          const double* invM, int s_num, int s_den, int s_rz_next, int s_rn);
// sums (a, b) and (a, c) over a 3n vector of a level into scal[s0], scal[s1] (c may be null)
int launch_dot2(hpc_ctx* c, int level, const double* a, const double* b, const double* cv, int s0, int s1);
int launch_dot2(hpc_ctx* c, int level, const float* a, const double* b, const double* cv, int s0, int s1);
// flexible direction p = z + beta p, beta = (scal[s_delta] - scal[s_gamma]) / scal[s_delta_prev]
// (Polak-Ribiere form of flexible CG), beta = 0 if first
int launch_fcg_dir(hpc_ctx* c, int level, const double* z, double* p, bool first, int s_delta, int s_gamma,
                   int s_delta_prev);
int launch_fcg_dir(hpc_ctx* c, int level, const float* z, double* p, bool first, int s_delta, int s_gamma,
                   int s_delta_prev);
int launch_pf_update(hpc_ctx* c, int level, const double* p, int s_rz, int s_pw, int s_rz_next, int s_rn);
// p = r M^-1 + beta p (beta = scal[s_rz]/scal[s_rz_prev], 0 if first), in place
int launch_dir_update(hpc_ctx* c, int level, int ncomp, const double* r, const double* invM, double* p, bool first,
                      int s_rz, int s_rz_prev);
// Dirichlet operations on a 3n vector of a level: kind 0 set u (Ut on top), 1 copy src into v,
// 2 zero v.
int launch_bc(hpc_ctx* c, int level, double* v, const double* src, int kind, double Ut);
// sum of squares of a 3n (ncomp=3) or n vector into scal[slot]; optional second vector for dots.
int launch_dot(hpc_ctx* c, int level, int ncomp, const double* a, const double* b, int slot);
// fill / copy helpers over padded levels
int launch_fill(hpc_ctx* c, double* v, long long n, double value);
// v = 1/v on the valid nodes of a level (ncomp components)
int launch_invert(hpc_ctx* c, int level, int ncomp, double* v);
cudaError_t kernel_binary_version(int* version);
int launch_axpby(hpc_ctx* c, double* y, const double* a, const double* b, double sa, double sb, long long n);
// Transfers
int launch_inject(hpc_ctx* c, int lf, const double* f, double* co, int ncomp);
int launch_inject_u(hpc_ctx* c, int lf, double Ut);  // u_c = u_f(2i), BC, uold_c = u_c (coarsen_u)
int launch_inject_d(hpc_ctx* c, int lf);             // d_c = d_f(2i), dold_c = d_c (coarsen_d)
int launch_restrict(hpc_ctx* c, int lf, const double* rf, const double* Fic, double* fc, int ncomp);
int launch_prolong(hpc_ctx* c, int lf, const double* uc, const double* ucold, double* uf, int ncomp,
                   bool apply_bc, double Ut);
// Material / history
int launch_choice_element(hpc_ctx* c, double small_k, bool do_choice, bool do_element);
int launch_vr(hpc_ctx* c, int lf, const double* Hf, double* Hc, bool hill, bool whole_array);
int launch_coarse_vr(hpc_ctx* c, int lf, const double* f, double* co);
int launch_strain_history(hpc_ctx* c, double lc, double uprop);
int launch_fd_h(hpc_ctx* c, int level);
int launch_dmax(hpc_ctx* c, int slot_dd, int slot_dmax, bool copy_old);
int launch_ue(hpc_ctx* c, double lc, int slot);
int launch_top_sum(hpc_ctx* c, int slot);
int launch_initial_crack(hpc_ctx* c, int level, double H_crack);
int launch_image_material(hpc_ctx* c, const uint8_t* dimage, const int* voxel_n, int ngray, const int* dgray,
                          const double* dE, const double* dnu, const double* dgc, double voxel_size);
int launch_mp_choice_level(hpc_ctx* c, int level);
int launch_choice_level(hpc_ctx* c, int level, double small_k, bool do_choice, bool do_element);
int launch_crack(hpc_ctx* c, int level, const uint8_t* fx, const uint8_t* fy, const uint8_t* fz, double Hc);
int launch_zero_count(hpc_ctx* c, int level, int ncomp, const double* v, int slot);
int upload_shape_table(const double* N64);
// Whole coarse-level pcg_u in one thread block (coarse_kernels.cu), for levels small enough
bool coarse_pcg_fits(hpc_ctx* c, int level);
int coarse_pcg_prepare();
int launch_coarse_pcg(hpc_ctx* c, int level, double Ut, int nb);
bool coarse_pcg_fits_geo(const LevelGeo& g);
int launch_coarse_pcg_on(hpc_ctx* c, const LevelGeo& g, double* u, const double* fu, double* ru, const double* invM,
                         const double* Ke, const double* Ge, double Ut, int nb);
int tuned_shapes(int* out5, int cap);  // measured strip shapes: {nx, ny, nz, wy, cz} per entry


// ---------------------------------------------------------------- solver pieces (hpcrack.cu) shared
// by the host-driven solves of hpc_step and the device-driven loops of hpc_batch_step
int check_zero_diags(hpc_ctx* c, int top, const char* what);
int mech_diags(hpc_ctx* c, int top, double small_k);
int pf_diags(hpc_ctx* c, int top, double lc);
int mech_diags_enqueue(hpc_ctx* c, int top, double small_k);
int pf_diags_enqueue(hpc_ctx* c, int top, double lc);
int mech_material(hpc_ctx* c, double small_k);
int gp_material(hpc_ctx* c, double small_k);
int cycle_u_top(hpc_ctx* c, const hpc_mg& mg, double small_k, double Ut, int t, bool allow_capture);
int cycle_d_top(hpc_ctx* c, const hpc_mg& mg, double lc, bool allow_capture);
int ensure_f32(hpc_ctx* c);
int f32_material(hpc_ctx* c);
int ensure_fcg(hpc_ctx* c);
int fcg_residual(hpc_ctx* c, double small_k, int t, int s_rn);
int fcg_iteration(hpc_ctx* c, const hpc_mg& mg, double small_k, int k, bool mixed, bool coarse_graph);
int voigt_all_level(hpc_ctx* c, int field);
int step_mid(hpc_ctx* c, const hpc_step_params* p);
int step_end(hpc_ctx* c, const hpc_step_params* p, int mcy, long long mit, int pcy, long long pit, double* out);
int step_end_enqueue(hpc_ctx* c);
int step_end_finish(hpc_ctx* c, const hpc_step_params* p, int mcy, long long mit, int pcy, long long pit, double* out);
int launch_set_scalar(hpc_ctx* c, int slot, double v);
int check_wait_error(hpc_ctx* c);

}  // namespace hpc
