/*
 * hpcrack.h - C ABI of the B200 library for HPCrack's staggered phase-field
 * fracture hot path (matrix-free FAS multigrid with restarted Jacobi-PCG
 * smoothers on trilinear-hex voxel grids).
 *
 * Every entry point returns an int status (HPC_OK = 0, see hpc_status); a
 * failing call leaves a message readable with hpc_last_error().  No entry point
 * falls back to the CPU: without a usable CUDA device hpc_create fails.
 *
 * Data layout seen by the caller is the reference's (include/grid.h:83-91):
 * one level of one field is a dense nx*ny*nz array of doubles, x fastest;
 * element (i,j,k) data live at node (i,j,k) of a node-sized array; level 0 is
 * the coarsest (include/mg.h:54-65).  Vector fields (u, fu, ru, uold) have
 * three components addressed by `comp`.  The library keeps device mirrors of
 * the whole hierarchy (gridded with an x pitch rounded up to 4 doubles) and
 * converts on hpc_upload / hpc_download.
 *
 * The reference has no FFI of its own: its interface is the set of C++ free
 * functions over grid<T>& / gdvec<T>& / mg<T>& declared in include/*.h of the
 * HPCrack project.  Each entry point below names the reference function it
 * replaces (path:line in the HPCrack project); the C++ drop-in shims in
 * hpcrack_b200/shim/ keep those exact signatures and call these functions.
 *
 * Threading: one host thread per context; all work of a context runs in order
 * on that context's CUDA stream.
 */
#ifndef HPCRACK_B200_H
#define HPCRACK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hpc_ctx hpc_ctx;

enum hpc_status {
  HPC_OK = 0,
  HPC_ERR_ARG = 1,        /* bad argument (level, field, size, null pointer) */
  HPC_ERR_CUDA = 2,       /* a CUDA runtime call failed */
  HPC_ERR_NOMEM = 3,      /* device allocation refused */
  HPC_ERR_DIVZERO = 4,    /* zero diagonal entry: the reference throws "Division by zero in grid /=
                             operation" (include/grid.h:182-190) */
  HPC_ERR_INPUT = 5,      /* gray level outside the material table, malformed input */
  HPC_ERR_NODEVICE = 6,   /* no CUDA device */
  HPC_ERR_IO = 7          /* an output file could not be opened or written */
};

/* Field ids (the reference's containers: crack_propagation.cpp:40-45, mechanical_displacement.cpp:
 * 28-35, phase_field.cpp:19-20). */
enum hpc_field {
  HPC_BULK = 0,   /* bulk modulus K, nodal, every level */
  HPC_G = 1,      /* shear modulus G, nodal */
  HPC_GC = 2,     /* fracture toughness Gc, nodal */
  HPC_D = 3,      /* phase field d */
  HPC_H = 4,      /* strain-history field H, element */
  HPC_FD = 5,     /* phase-field right-hand side */
  HPC_KE = 6,     /* element bulk modulus K_element */
  HPC_GE = 7,     /* element shear modulus G_element */
  HPC_R = 8,      /* phase-field residual */
  HPC_DOLD = 9,   /* coarse-level d saved at injection */
  HPC_DOLDF = 10, /* finest d of the previous increment (d_old) */
  HPC_U = 16,     /* displacement, 3 components */
  HPC_FU = 17,    /* mechanical right-hand side / reactions */
  HPC_RU = 18,    /* mechanical residual */
  HPC_UOLD = 19,  /* coarse-level u saved at injection */
  HPC_CHOICE = 32 /* regime 0/1/2 per element (int16 on the host side) */
};

typedef struct {
  int maxlevel;          /* finest level index; level 0 is the coarsest */
  int element_nb[3];     /* elements per axis on the coarsest level (config element_nb) */
  double x_start[3];     /* domain origin (config X_start) */
  int roi_start[3];      /* image ROI start (config ROI_start_*) */
} hpc_geometry;

/* Multigrid parameters, the reference's MG struct (include/mg.h:18-25). */
typedef struct {
  int nu0, nu1, nu2, gamma, ncy;
} hpc_mg;

/* One staggered load increment (crack_propagation.cpp:65-121) with its constants as parameters. */
typedef struct {
  int t;               /* increment index; t == 0 sets f_norm from reactions and Ue */
  hpc_mg mg_u, mg_d;
  double small_k;      /* residual stiffness k (crack_propagation.cpp:32) */
  double lc;           /* phase-field length scale l (already multiplied by h, main.cpp:94) */
  double voxel_size;   /* reaction scaling (crack_propagation.cpp:96) */
  double ut0;          /* <= 0: Ut0 = Ue (U_e) and dU = du_factor * Ue, as the reference */
  double du;           /* load step when ut0 > 0 */
  double du_factor;    /* 1.5e-3 in the reference (crack_propagation.cpp:76) */
  double mech_tol;     /* squared ratio |r|^2/|f|^2 (1e-6 in mechanical_displacement.cpp:88) */
  double pf_tol;       /* squared tests of phase_field.cpp:30-43 (1e-12 there) */
  int mech_solver;     /* HPC_MECH_FAS (0): the reference's FAS V-cycles (plain form);
                          HPC_MECH_FCG (1): flexible PCG preconditioned by one FP64 V-cycle;
                          HPC_MECH_MIXED (2): the precision form, the same with the V-cycle in FP32
                          (coarsest solve FP64); see hpc_u_entire_fcg */
} hpc_step_params;

enum { HPC_MECH_FAS = 0, HPC_MECH_FCG = 1, HPC_MECH_MIXED = 2 };

/* ---------------- context ---------------- */

/* Allocates the device mirrors of the whole hierarchy on `device` (initialize, initialization.cpp:
 * 19-134, and the mg / mgvec containers of crack_propagation.cpp:40-45).  The memory comes from the
 * device's default stream-ordered pool, in the order of the context's stream; the first context on a
 * device raises that pool's release threshold, so memory a destroyed context returns stays with the
 * process for the next context instead of going back to the driver (creating and destroying
 * contexts while others run synchronises nothing). */
int hpc_create(hpc_ctx** out, const hpc_geometry* geo, int device);
int hpc_destroy(hpc_ctx* ctx);
/* Device bytes a context of this geometry holds at most while it solves (admission by HBM
 * footprint): what hpc_create allocates plus everything allocated on first use by the solves, the
 * precision form, checkpoints and uploads.  Not included: the VTK character buffers of
 * hpc_vtk_write (up to 16 bytes per node of the written level) and the tensor-core kernel's
 * per-block tensor memory. */
int hpc_footprint(const hpc_geometry* geo, size_t* bytes);
/* Level geometry as initialize() builds it (initialization.cpp:19-134). */
int hpc_level_dims(hpc_ctx* ctx, int level, int* n3, double* h3);
int hpc_sync(hpc_ctx* ctx);
const char* hpc_last_error(void);
/* 1 (default) reproduces the reference's MP_choice loop bounds (material_selection.cpp:60-63),
 * 0 visits every element. */
int hpc_set_choice_quirk(hpc_ctx* ctx, int reproduce);
/* No counterpart in the reference: 1 makes this context measure the strip shape (element rows x
 * planes per warp) of each element kernel on each level size at its first use, by timing the
 * candidates on the live data, instead of taking the latency model's choice; measured shapes are
 * shared by every context of the process.  Results differ from the model's shapes only in the
 * rounding of the reductions (the grid changes); the default 0 keeps runs reproducible. */
int hpc_set_autotune(hpc_ctx* ctx, int on);
/* The measured shapes so far: up to cap entries {nx, ny, nz, element rows, planes}. */
int hpc_tuned_shapes(int* out5, int cap, int* count);
/* No counterpart in the reference: 1 (default) runs pcg_u on the coarsest level (mechanical_pcg.cpp:
 * 223-330 as called by mechanical_multigrid.cpp:29-32) in one thread block when the level fits in
 * shared memory (up to about 10^3 nodes); 0 uses the per-iteration kernels.  The two differ only in
 * the order of the same sums. */
int hpc_set_fused_coarsest(hpc_ctx* ctx, int on);
/* No counterpart in the reference: 1 runs the element operator of the precision form's FP32 V-cycle
 * (mech_solver HPC_MECH_MIXED) on the tensor cores - strains and element forces as two TF32 GEMMs
 * per 128 elements (tcgen05, accumulators in tensor memory), Hooke's law per Gauss point on the
 * CUDA cores - on levels with equal spacing in x, y and z; 0 (default) keeps the FP32 stencil
 * kernels.  TF32 operands approximate the FP32 operator to about 1e-3; the flexible PCG around the
 * V-cycle keeps its FP64 residual, so the solution meets the same tolerance. */
int hpc_set_tensor_apply(hpc_ctx* ctx, int on);
/* No counterpart in the reference: 1 stages the node rows of the finest-level operator applies
 * (FP64 and the precision form's FP32, with the Gauss-point moduli of a mechanical solve) with
 * tensor-memory-accelerator copies - one cp.async.bulk.tensor per row of three components on two
 * planes, completion on an mbarrier - instead of per-lane cp.async (the default); 0 stages with
 * per-lane cp.async.  The same values reach the same arithmetic: the same bits. */
int hpc_set_tma_staging(hpc_ctx* ctx, int on);
/* Kernels launched by this context since the last reset (instrumentation for benchmarks). */
int hpc_launch_count(hpc_ctx* ctx, long long* count, int reset);
/* The context's CUDA stream (cudaStream_t), for callers that time on it. */
void* hpc_stream(hpc_ctx* ctx);
/* No counterpart in the reference: the compute capability the library's device code was built for,
 * as the CUDA runtime reports it for one of the library's kernels on the current device
 * (major * 10 + minor: 100 for sm_100a).  HPC_ERR_NODEVICE without a device. */
int hpc_binary_version(int* version);
/* Kernel classes that can be timed with CUDA events on the context's stream. */
enum hpc_kernel_class {
  HPC_KC_NONE = -1,
  HPC_KC_MECH_PCG_FINEST = 0,   /* w = K(d) p and (p, w) on the finest level (FP64) */
  HPC_KC_PF_PCG_FINEST = 1,     /* w = A_d p and (p, w) on the finest level */
  HPC_KC_MECH_UPDATE_FINEST = 2, /* u += alpha p, r -= alpha w, rz and |r|^2 on the finest level */
  HPC_KC_MECH32_PCG_FINEST = 3   /* the precision form's FP32 w = K p on the finest level */
};
/* Records a start/stop event pair around every launch of `kernel_class` from now on (HPC_KC_NONE
 * stops recording); resets the record. */
int hpc_kernel_timing(hpc_ctx* ctx, int kernel_class);
/* Synchronises and returns the number of recorded launches and their summed device time (ms). */
int hpc_kernel_time(hpc_ctx* ctx, long long* launches, double* total_ms);

/* ---------------- host <-> device (dense x-fastest host arrays) ---------------- */
/* Both return when the copy is complete.  The first upload allocates a dense finest-size device
 * buffer (8 bytes per finest node, counted by hpc_footprint): an upload is one contiguous copy into it
 * and a kernel that spreads it into the padded layout. */
int hpc_upload(hpc_ctx* ctx, int field, int level, int comp, const double* host);
int hpc_download(hpc_ctx* ctx, int field, int level, int comp, double* host);
int hpc_upload_choice(hpc_ctx* ctx, int level, const int16_t* host);
int hpc_download_choice(hpc_ctx* ctx, int level, int16_t* host);
/* Loop state of the staggered driver: {f_norm, fd_norm, Ue, Ut, dU, u_proportion}. */
int hpc_get_state(hpc_ctx* ctx, double* s6);
int hpc_set_state(hpc_ctx* ctx, const double* s6);

/* ---------------- checkpoint / restart ---------------- */
/* The history dumps of crack_propagation.cpp:99-106 (write_vector_3D of u, v, w, H, d,
 * write_read_history.cpp:18-53) made restartable: the finest u (3 components), H, d and d_old plus
 * the loop state are snapshotted on the device (dense x-fastest, the reference's file order) and
 * copied to pinned host memory on a separate stream, overlapping the increments that follow.  The
 * first call allocates 6 dense finest-level arrays on the device and in pinned host memory. */
int hpc_checkpoint_begin(hpc_ctx* ctx, int t);
/* Waits for the copy of the last hpc_checkpoint_begin.  *fields points to 6 consecutive dense
 * arrays of nx*ny*nz doubles (u, v, w, H, d, d_old), valid until the next hpc_checkpoint_begin or
 * hpc_destroy; state6 as hpc_get_state at the time of the snapshot; *t the index given to begin.
 * Each output may be null. */
int hpc_checkpoint_wait(hpc_ctx* ctx, int* t, const double** fields, double* state6);
/* Restores a checkpoint into the finest level (read_vector_3D, write_read_history.cpp:55-86, for
 * the fields) and the loop state; the next hpc_step continues as the uninterrupted run would. */
int hpc_checkpoint_restore(hpc_ctx* ctx, const double* u, const double* v, const double* w, const double* H,
                           const double* d, const double* d_old, const double* state6);

/* ---------------- VTK output ---------------- */
/* write_total_de / write_total_u / write_total_H (vtk_output.cpp:420-469) of one rank: the .vti
 * piece (Float32 values, base64, XML ImageData) and the .pvti index of one field of one level,
 * byte-identical to the reference's files.  option "S": scalar point data (a scalar field), "V":
 * vector point data (a vector field, every value multiplied by `scale` first, as write_vector does
 * with u_proportion), "C": cell data of the element slots (write_celltdata_H).  Paths follow
 * open_file / write_pvtk (vtk_output.cpp:26-35, :362-367): Output/<filename>_l_<level>_t_<t>_Proc_0.vti
 * and Output/<filename>_l_<level>_t_<t>.pvti unless filename contains ".vti" / ".pvti"; the Output
 * folder must exist.  The field is converted and encoded on the device on the context's stream,
 * copied to pinned host memory on a copy stream and written by a host thread, so the call returns
 * at once and later work on the context overlaps the copy and the writes; the first call allocates
 * the character buffers (16 bytes per node for "V", 16/3 for "S"), on the device and in pinned host
 * memory.  One write is in flight per context: a second call first waits for the previous one.
 * The reference's combined "VS" writer (write_total_Eu) is not offered: its file lacks the second
 * DataArray's opening tag. */
int hpc_vtk_write(hpc_ctx* ctx, const char* option, int field, int level, double scale, const char* filename,
                  const char* field_name, int t);
/* Waits for the write in flight; returns its status (HPC_ERR_IO if a file could not be written). */
int hpc_vtk_wait(hpc_ctx* ctx);

/* ---------------- operators ---------------- */
/* Internal_Force: dst = K(d) src on one level (mechanical_pcg.cpp:174-191). */
int hpc_internal_force(hpc_ctx* ctx, int level, int src_field, int dst_field, double small_k);
/* PreM_u: dst = diag K(d) (mechanical_pcg.cpp:102-112). */
int hpc_prem_u(hpc_ctx* ctx, int level, int dst_field, double small_k);
/* Fld: dst = A_d src (phase_field_pcg.cpp:93-103). */
int hpc_fld(hpc_ctx* ctx, int level, int src_field, int dst_field, double lc);
/* Precondition_M: dst = diag A_d (phase_field_pcg.cpp:49-59). */
int hpc_precondition_m(hpc_ctx* ctx, int level, int dst_field, double lc);

/* ---------------- smoothers, cycles, solves ---------------- */
/* Initial_residual_u (mechanical_pcg.cpp:193-220). */
int hpc_initial_residual_u(hpc_ctx* ctx, int level, double small_k, double* r_norm);
/* pcg_u (mechanical_pcg.cpp:223-330; declared mechanical_pcg.h:47-51). */
int hpc_pcg_u(hpc_ctx* ctx, int level, double small_k, double Ut, int nb_relax, int t, double* f_norm);
/* initial_residual (phase_field_pcg.cpp:106-131). */
int hpc_initial_residual_d(hpc_ctx* ctx, int level, double lc, double* r_norm);
/* pcg_d (phase_field_pcg.cpp:133-214; declared phase_field_pcg.h:36-38). */
int hpc_pcg_d(hpc_ctx* ctx, int level, double lc, int nb_relax, int t, double* fd_norm);
/* cycle_u (mechanical_multigrid.cpp:18-54). */
int hpc_cycle_u(hpc_ctx* ctx, int level, const hpc_mg* mg, double small_k, double Ut, int t, double* f_norm);
/* cycle_d (phase_field_multigrid.cpp:18-44). */
int hpc_cycle_d(hpc_ctx* ctx, int level, const hpc_mg* mg, double lc, int t, double* fd_norm);
/* u_entire (mechanical_displacement.cpp:25-115): cycles and finest smoother iterations returned. */
int hpc_u_entire(hpc_ctx* ctx, const hpc_mg* mg, double small_k, double Ut, int t, double* f_norm,
                 double mech_tol, int* cycles, int* iters);
/* phase_field (phase_field.cpp:15-57). */
int hpc_phase_field(hpc_ctx* ctx, const hpc_mg* mg, double lc, int t, double* fd_norm, double pf_tol,
                    int* cycles, int* iters);
/* No counterpart in the reference: the mechanical solve of u_entire (mechanical_displacement.cpp:25-115)
 * by flexible PCG on the finest level (true residual, dot products and updates in FP64),
 * preconditioned by one V-cycle of cycle_u's kind per iteration, in FP64 (mixed = 0) or on
 * single-precision copies of the levels with an FP64 coarsest solve (mixed = 1, the precision form);
 * same stopping test |r|^2/|f|^2 <= mech_tol, f_norm from the reactions at t == 0, reactions into
 * fu at the end.  *cycles = outer iterations (= V-cycles), *iters = finest smoother iterations. */
int hpc_u_entire_fcg(hpc_ctx* ctx, const hpc_mg* mg, double small_k, double Ut, int t, double* f_norm,
                     double mech_tol, int mixed, int* cycles, int* iters);
/* One staggered increment (crack_propagation.cpp:65-121).  out[8] = {Ut, F (u_proportion*FeW),
 * delta_d_max, d_max, mech cycles, pf cycles, mech finest iters, pf finest iters}. */
int hpc_step(hpc_ctx* ctx, const hpc_step_params* p, double* out);

/* ---------------- material, history, reductions ---------------- */
/* MP_choice (material_selection.cpp:47-65). */
int hpc_mp_choice(hpc_ctx* ctx);
/* MP_all_element (material_selection.cpp:100-116). */
int hpc_mp_all_element(hpc_ctx* ctx, double small_k);
/* VR_all_level (material_coarse_element.cpp:86-102). */
int hpc_vr_all_level(hpc_ctx* ctx, int field);
/* Voigt_all_level (material_coarse_element.cpp:106-118). */
int hpc_voigt_all_level(hpc_ctx* ctx, int field);
/* coarse_VR (image_input.cpp:244-260). */
int hpc_coarse_vr(hpc_ctx* ctx, int field);
/* strain_history (strain_history.cpp:162-210). */
int hpc_strain_history(hpc_ctx* ctx, double lc, double u_proportion);
/* fd_h (phase_field_right_hand_side.cpp:14-47). */
int hpc_fd_h(hpc_ctx* ctx, int level);
/* delta_d_max / d_max (phase_field_max_search.cpp:17-53). */
int hpc_delta_d_max(hpc_ctx* ctx, double* out);
int hpc_d_max(hpc_ctx* ctx, double* out);
/* U_e (strain_history.cpp:86-131). */
int hpc_U_e(hpc_ctx* ctx, double lc, double* out);
/* externe_force_nodal / externe_force_sum (mechanical_right_hnd.cpp:18-59). */
int hpc_externe_force_nodal(hpc_ctx* ctx, double Ut, double small_k);
int hpc_externe_force_sum(hpc_ctx* ctx, double* out);
/* initial_crack (strain_history.cpp:30-70). */
int hpc_initial_crack(hpc_ctx* ctx, double H_crack, int level);

/* ---------------- boundary conditions (boundary_conditions.cpp:20-154) ---------------- */
int hpc_dirichlet_bd(hpc_ctx* ctx, int level, int field, double Ut);
int hpc_dirichlet_force(hpc_ctx* ctx, int level, int f_field, int fi_field);
int hpc_dirichlet_residual(hpc_ctx* ctx, int level, int field);

/* ---------------- inter-grid transfers (multigrid_intergrid.cpp) ---------------- */
/* solution_injection (:25-90): level lf-1 of `field` from level lf. */
int hpc_solution_injection(hpc_ctx* ctx, int field, int comp, int lf);
/* coarsen_f_standard_routine (:124-342): fc(lf-1) = Fic(lf-1) + full weighting of rf(lf). */
int hpc_coarsen_f_standard(hpc_ctx* ctx, int fc_field, int rf_field, int fic_field, int comp, int lf);
/* refine_standard_routine (:416-520): uf(lf) += P (uc(lf-1) - ucold(lf-1)). */
int hpc_refine_standard(hpc_ctx* ctx, int uf_field, int uc_field, int ucold_field, int comp, int lf);

/* ---------------- input path (image_input.cpp:120-282, csv_reader.cpp) ---------------- */
/* Raw uint8 image (x fastest, voxel_n[3] voxels) + gray-level table -> finest bulK, G, gc, then the
 * nodal Voigt-Reuss-Hill hierarchy (coarse_VR). */
int hpc_image_material(hpc_ctx* ctx, const uint8_t* image, const int* voxel_n, int ngray, const int* gray,
                       const double* E, const double* nu, const double* gc, double voxel_size);

/* ---------------- batched increments ---------------- */
/* No counterpart in the reference (it runs one specimen per program): a batch advances many contexts
 * (specimens of any sizes, on one device) by one staggered increment each - the loop body of
 * crack_propagation.cpp:65-121, as hpc_step does for one context.  Each specimen's mechanical solve
 * (any mech_solver) and phase-field solve is a device-driven loop: one CUDA graph per batch holds,
 * for every specimen, a conditional WHILE node whose body is the specimen's V-cycle (or flexible-PCG
 * iteration) and a kernel applying the reference's stopping rule, so one graph launch runs every
 * specimen's solve to its own convergence (at most ncy cycles).  Results are bit-identical to
 * hpc_step on each context alone.  The graphs are kept and reused while the batch's composition and
 * the specimens' loop parameters stay the same, and rebuilt before a call with any other composition
 * runs, so a context may be destroyed once the call that ran it has returned.  One calling thread per
 * batch. */
typedef struct hpc_batch hpc_batch;
int hpc_batch_create(hpc_batch** out);
int hpc_batch_destroy(hpc_batch* batch);
/* ctxs[0..n): distinct contexts on one device; params[i] drives ctxs[i] (its own t, tolerances, mg
 * parameters, mech_solver); out[8 i .. 8 i + 8) receives what hpc_step writes for ctxs[i]. */
int hpc_batch_step(hpc_batch* batch, hpc_ctx* const* ctxs, int n, const hpc_step_params* params, double* out);
/* No counterpart in the reference: cumulative instrumentation of a batch - out[0] host seconds spent
 * enqueuing and reading outside graph builds and waits, out[1] seconds building graphs, out[2]
 * seconds waiting for the graphs (only measured while waits are on), out[3] graph builds, out[4]
 * graph launches.  on = 1 makes every hpc_batch_step wait for each graph right after its launch (to
 * time it), 0 turns that off, -1 leaves it as it is; out may be null. */
int hpc_batch_timing(hpc_batch* batch, int on, double* out);

/* ---------------- allocation-free variant ---------------- */
/* No counterpart in the reference: d_max and delta_d_max (the reductions of hpc_d_max /
 * hpc_delta_d_max) of caller-owned DEVICE arrays d and d_old of n doubles, written to the caller's
 * device array out[2] = {max(0, max(d - d_old)), max(0, max d)}, on `stream` (a cudaStream_t, may
 * be null).  For callers that cannot allocate device memory (an allocator that owns the device,
 * code that must not trigger cudaMalloc's implicit synchronisation): the block partials live in a
 * fixed 1 MiB __device__ array that every device loading the library keeps until exit, so the call
 * allocates nothing.  n is limited to 134217728 (HPC_ERR_ARG beyond).  The first call on a device
 * looks up the scratch address once; under lazy module loading (the CUDA 12 default) that lookup
 * can load the library's device code and so allocate and synchronise: make one warm-up call (or any
 * other call of this library on that device) before a region that must not allocate and before
 * any stream capture.  The cached address does not survive cudaDeviceReset.  All calls share the
 * scratch: calls that overlap on the GPU race. */
int hpc_dmax_noalloc(const double* d, const double* d_old, long long n, double* out, void* stream);

/* ---------------- one specimen split along z over ranks ---------------- */
/* The reference's MPI domain decomposition (3-D, MPI_Cart) restricted to z, one rank per GPU or per
 * host thread.  Replaces, for a z-split:
 *   - the per-rank level sizes of initialize (initialization.cpp:19-134): coarsest nodes
 *     q = (kk + 1) / nranks per rank, the last rank also the remainder, one ghost plane on every
 *     side that has a neighbour;
 *   - the rank's coordinates, get_coordinate (boundary_conditions.cpp:13-18): the Dirichlet sets,
 *     the image planes and the pre-crack are those of the whole specimen;
 *   - realdomain (realdomain.h:17-40): vv_product / grid_norm (pcg_utilities.cpp:16-58), d_max,
 *     delta_d_max (phase_field_max_search.cpp:17-53) and the reaction sum
 *     (mechanical_right_hnd.cpp:40-59) run over owned planes and are combined over the ranks;
 *   - SendRecv (mpi_communications.h:24-47) in z at the reference's call sites: after the PCG
 *     direction (mechanical_pcg.cpp:278, phase_field_pcg.cpp:180), injection
 *     (multigrid_intergrid.cpp:99,116), before the restriction (:356,393), after prolongation
 *     (:531,547) and after the coarse material (image_input.cpp:269,
 *     material_coarse_element.cpp:98,114).
 * A slab context holds only its planes: hpc_upload / hpc_download / hpc_level_dims see the local
 * nx * ny * nz_local arrays (ghost planes included).  Every call that solves, transfers or reduces
 * is a collective step: all ranks make the same calls in the same order.  A slab runs every
 * mech_solver of hpc_step (hpc_batch_step returns HPC_ERR_ARG; the precision form's element
 * contraction stays on the CUDA cores), without strip autotuning; the coarse parts of its cycles replay as CUDA graphs
 * over NCCL (the NCCL calls captured inside), not over the in-process transport.  Its coarsest level is gathered on
 * every rank and solved redundantly by the one-block solver when the whole level fits it (one
 * exchange per visit instead of three collective steps per iteration; hpc_set_fused_coarsest(ctx, 0)
 * selects the reference's distributed smoother there).
 * Out of scope: x and y splits. */
/* Host only, no device: out4 = {local nz, global z index of local plane 0, first owned plane, one
 * past the last owned plane} of rank `rank` of `nranks` on `level`; HPC_ERR_ARG if a rank would own
 * no coarsest plane. */
int hpc_slab_level(const hpc_geometry* geo, int nranks, int rank, int level, int* out4);
/* A context for rank `rank` of `nranks`; it joins a transport before its first collective step.  The
 * 2^31-node limit of hpc_create applies to each rank's planes, so a split specimen may exceed it (and
 * one GPU's memory). */
int hpc_create_slab(hpc_ctx** out, const hpc_geometry* geo, int device, int nranks, int rank);
/* hpc_footprint of rank `rank`'s slab (its planes, and the whole coarsest level it gathers). */
int hpc_footprint_slab(const hpc_geometry* geo, int nranks, int rank, size_t* bytes);
/* In-process transport: the ranks are host threads of this process (each calling its own context,
 * all at once), on one device or several; planes move by device copies, reductions are combined
 * on the host in rank order (every rank gets the same bits).  A wait for a rank that does not
 * arrive ends after 120 s with HPC_ERR_CUDA; hpc_slab_group_abort ends every wait at once.  The
 * group outlives its member contexts. */
typedef struct hpc_slab_group hpc_slab_group;
int hpc_slab_group_create(hpc_slab_group** out, int nranks);
int hpc_slab_group_join(hpc_slab_group* group, hpc_ctx* ctx);
int hpc_slab_group_abort(hpc_slab_group* group);
int hpc_slab_group_destroy(hpc_slab_group* group);
/* NCCL transport, one process per GPU: rank 0 makes the id, the caller hands it to every rank (a
 * torch.distributed broadcast, a file), each rank joins with its context (ncclCommInitRank: all
 * ranks at once).  NCCL is loaded at run time (libnccl.so.2); HPC_ERR_NODEVICE without it. */
int hpc_nccl_unique_id(unsigned char* out128);
int hpc_slab_join_nccl(hpc_ctx* ctx, const unsigned char* id128);

#ifdef __cplusplus
}
#endif
#endif
