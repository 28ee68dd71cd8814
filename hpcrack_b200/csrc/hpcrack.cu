// Host side of the B200 HPCrack library: context and device hierarchy, host<->device transfers,
// the solver drivers (restarted Jacobi-PCG smoothers, FAS V-cycles, the mechanical and
// phase-field solves, one staggered increment) and the C ABI of include/hpcrack.h.
//
// The drivers issue kernels on the context's stream; the PCG scalars (rz, pw, alpha, beta) never
// leave the device.  The host synchronises once per V-cycle (to test convergence, exactly where
// the reference tests it) and at the end of a call.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace hpc {

// ---------------------------------------------------------------- errors
static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
int cuda_fail(cudaError_t e, const char* where) {
  g_err = std::string(where) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return HPC_ERR_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return HPC_ERR_NODEVICE;
  return HPC_ERR_CUDA;
}
static int arg_fail(const std::string& msg) {
  g_err = msg;
  return HPC_ERR_ARG;
}

// ---------------------------------------------------------------- context memory
// A context's device memory comes from the device's stream-ordered pool, allocated and released in
// the order of the context's stream: releasing a finished request's memory does not synchronise the
// whole device (cudaFree does) while other contexts run, and the pool keeps it for the next request
// (release threshold raised once per device: the memory stays with the process).
void pool_setup(int device) {
  static std::mutex mu;
  static bool done[64] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= 64 || done[device]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done[device] = true;
}
cudaError_t ctx_alloc(hpc_ctx* c, void** p, size_t bytes) { return cudaMallocAsync(p, bytes, c->stream); }
void ctx_free(hpc_ctx* c, void* p) {
  if (p) cudaFreeAsync(p, c->stream);
}

// Pinned host slots for the contexts' scalar reads (64 doubles each), carved from chunks allocated
// once per process: creating and destroying contexts allocates and frees no pinned memory (cudaFreeHost
// synchronises the device).
static std::mutex g_pin_mu;
static std::vector<double*> g_pin_free;
static double* pinned_slot() {
  std::lock_guard<std::mutex> lock(g_pin_mu);
  if (g_pin_free.empty()) {
    constexpr int kSlots = 256;
    double* chunk = nullptr;
    if (cudaMallocHost((void**)&chunk, sizeof(double) * 64 * kSlots) != cudaSuccess) return nullptr;
    for (int i = kSlots - 1; i >= 0; --i) g_pin_free.push_back(chunk + 64 * i);
  }
  double* p = g_pin_free.back();
  g_pin_free.pop_back();
  return p;
}
static void pinned_release(double* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_pin_mu);
  g_pin_free.push_back(p);
}

void timing_begin(hpc_ctx* c, int cls) {
  if (cls < 0 || cls != c->timing_class) return;
  if (c->tev_used >= c->tev_cap) {
    const int cap = c->tev_cap ? 2 * c->tev_cap : 256;
    cudaEvent_t* ev = new cudaEvent_t[2 * cap];
    for (int i = 0; i < 2 * c->tev_cap; ++i) ev[i] = c->tev[i];
    for (int i = 2 * c->tev_cap; i < 2 * cap; ++i) cudaEventCreate(&ev[i]);
    delete[] c->tev;
    c->tev = ev;
    c->tev_cap = cap;
  }
  cudaEventRecord(c->tev[2 * c->tev_used], c->stream);
}
void timing_end(hpc_ctx* c, int cls) {
  if (cls < 0 || cls != c->timing_class || c->tev_used >= c->tev_cap) return;
  cudaEventRecord(c->tev[2 * c->tev_used + 1], c->stream);
  c->tev_used++;
}

// ---------------------------------------------------------------- geometry
struct HostLevel {
  int nx, ny, nz, px;
  double hx, hy, hz;
};

// input_setting (image_input.cpp:21-27) and initialize (initialization.cpp:19-134) for one rank.
static void host_geometry(const hpc_geometry& g, double box[6], HostLevel* lv) {
  int coefb[3];
  for (int a = 0; a < 3; ++a) coefb[a] = (int)(g.roi_start[a] + g.element_nb[a] * std::pow(2, g.maxlevel));
  box[0] = g.x_start[0];
  box[1] = g.x_start[0] + coefb[0];
  box[2] = g.x_start[1];
  box[3] = g.x_start[1] + coefb[1];
  box[4] = g.x_start[2];
  box[5] = g.x_start[2] + coefb[2];
  double hx = (box[1] - box[0]) / g.element_nb[0];
  double hy = (box[3] - box[2]) / g.element_nb[1];
  double hz = (box[5] - box[4]) / g.element_nb[2];
  int nx = g.element_nb[0] + 1, ny = g.element_nb[1] + 1, nz = g.element_nb[2] + 1;
  for (int l = 0; l <= g.maxlevel; ++l) {
    lv[l].nx = nx;
    lv[l].ny = ny;
    lv[l].nz = nz;
    lv[l].px = (nx + kPitchAlign - 1) / kPitchAlign * kPitchAlign;
    lv[l].hx = hx;
    lv[l].hy = hy;
    lv[l].hz = hz;
    hx *= 0.5;
    hy *= 0.5;
    hz *= 0.5;
    nx = 2 * (nx - 1) + 1;
    ny = 2 * (ny - 1) + 1;
    nz = 2 * (nz - 1) + 1;
  }
}

// The geometry of rank r of nr along z (one rank: the whole specimen).
static bool geometry_ok(const hpc_geometry* g, int nr = 1, int r = 0) {
  if (!g || g->maxlevel < 0 || g->maxlevel >= kMaxLevels) return false;
  for (int a = 0; a < 3; ++a)
    if (g->element_nb[a] < 1 || g->roi_start[a] < 0) return false;
  // finest node count per axis must stay a sane int
  for (int a = 0; a < 3; ++a)
    if ((double)g->element_nb[a] * std::pow(2.0, g->maxlevel) > 65000.0) return false;
  SlabLevel sl[kMaxLevels];
  if (!slab_levels(*g, nr, r, sl)) return false;
  // node-parallel kernels index a level with 32-bit arithmetic: padded node count of the planes this
  // context holds below 2^31 (a split lets a specimen exceed that, each rank's slab may not)
  double nodes = (double)sl[g->maxlevel].nz;
  for (int a = 0; a < 2; ++a) nodes *= (double)g->element_nb[a] * std::pow(2.0, g->maxlevel) + 1.0 + (a == 0 ? 3 : 0);
  if (nodes >= 2147483648.0) return false;
  return true;
}

// Number of doubles per level allocated for a level with n padded slots.
constexpr int kScalarFieldsPerLevel = 10;  // bulK G gc d H fd Ke Ge R dold
constexpr int kVectorFieldsPerLevel = 4;   // u fu ru uold
constexpr int kWork3 = 4, kWork1 = 4;      // preMu p w tmp3 / preMd pd wd tmp1
static size_t level_bytes(long long n) {
  return (size_t)n * sizeof(double) * (kScalarFieldsPerLevel + 3 * kVectorFieldsPerLevel + 3 * kWork3 + kWork1) +
         (size_t)n;  // choice
}

double* scalar_field(hpc_ctx* c, int field, int level) {
  if (level < 0 || level > c->maxlevel) return nullptr;
  LevelFields& F = c->F[level];
  switch (field) {
    case HPC_BULK: return F.bulK;
    case HPC_G: return F.G;
    case HPC_GC: return F.gc;
    case HPC_D: return F.d;
    case HPC_H: return F.H;
    case HPC_FD: return F.fd;
    case HPC_KE: return F.Ke;
    case HPC_GE: return F.Ge;
    case HPC_R: return F.R;
    case HPC_DOLD: return F.dold;
    case HPC_DOLDF: return level == c->maxlevel ? c->d_old : nullptr;
    default: return nullptr;
  }
}
double* vector_field(hpc_ctx* c, int field, int level) {
  if (level < 0 || level > c->maxlevel) return nullptr;
  LevelFields& F = c->F[level];
  switch (field) {
    case HPC_U: return F.u;
    case HPC_FU: return F.fu;
    case HPC_RU: return F.ru;
    case HPC_UOLD: return F.uold;
    default: return nullptr;
  }
}
static double* component(hpc_ctx* c, int field, int level, int comp) {
  if (double* s = scalar_field(c, field, level)) return comp == 0 ? s : nullptr;
  if (double* v = vector_field(c, field, level)) return (comp >= 0 && comp < 3) ? v + (size_t)comp * c->L[level].n : nullptr;
  return nullptr;
}

int read_scalars(hpc_ctx* c, int first, int count, double* out) {
  HPC_CUDA(cudaMemcpyAsync(c->hscal, c->scal + first, sizeof(double) * count, cudaMemcpyDeviceToHost, c->stream));
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  std::memcpy(out, c->hscal, sizeof(double) * count);
  return HPC_OK;
}
int write_scalar(hpc_ctx* c, int slot, double v) {
  // stage through the pinned buffer's tail so the async copy has a stable source
  c->hscal[63] = v;
  HPC_CUDA(cudaMemcpyAsync(c->scal + slot, c->hscal + 63, sizeof(double), cudaMemcpyHostToDevice, c->stream));
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  return HPC_OK;
}

// N(g, n) exactly as Dshape_function computes it (shape_function.cpp:16-75), for fd_h.
static void shape_table(double N[64]) {
  double x[8] = {-1., 1., 1., -1., -1., 1., 1., -1.};
  double y[8] = {-1., -1., 1., 1., -1., -1., 1., 1.};
  double z[8] = {-1., -1., -1., -1., 1., 1., 1., 1.};
  for (int i = 0; i < 8; i++) {
    x[i] = x[i] / std::sqrt(3);
    y[i] = y[i] / std::sqrt(3);
    z[i] = z[i] / std::sqrt(3);
    N[i * 8 + 0] = 0.125 * (1 - x[i]) * (1 - y[i]) * (1 - z[i]);
    N[i * 8 + 1] = 0.125 * (1 + x[i]) * (1 - y[i]) * (1 - z[i]);
    N[i * 8 + 2] = 0.125 * (1 + x[i]) * (1 + y[i]) * (1 - z[i]);
    N[i * 8 + 3] = 0.125 * (1 - x[i]) * (1 + y[i]) * (1 - z[i]);
    N[i * 8 + 4] = 0.125 * (1 - x[i]) * (1 - y[i]) * (1 + z[i]);
    N[i * 8 + 5] = 0.125 * (1 + x[i]) * (1 - y[i]) * (1 + z[i]);
    N[i * 8 + 6] = 0.125 * (1 + x[i]) * (1 + y[i]) * (1 + z[i]);
    N[i * 8 + 7] = 0.125 * (1 - x[i]) * (1 + y[i]) * (1 + z[i]);
  }
}

// ---------------------------------------------------------------- solver drivers
static bool is_finest(hpc_ctx* c, int l) { return l == c->maxlevel; }

// Every level's zero-diagonal count goes to its own slot; one read checks them all.
int check_zero_diags(hpc_ctx* c, int top, const char* what) {
  double z[kMaxLevels];
  int rc = read_scalars(c, S_ZEROS, top + 1, z);
  if (rc) return rc;
  for (int l = 0; l <= top; ++l)
    if (z[l] > 0) {
      set_error(std::string("zero diagonal entry in ") + what + ": Division by zero in grid /= operation");
      return HPC_ERR_DIVZERO;
    }
  return HPC_OK;
}

// diag K(d) of every level 0..top into preMu; fails like the reference on a zero entry.
// The diagonals without the zero check (check_zero_diags reads the counts: a host synchronisation).
int mech_diags_enqueue(hpc_ctx* c, int top, double small_k) {
  for (int l = 0; l <= top; ++l) {
    int rc = launch_mech_diag(c, l, is_finest(c, l), small_k, c->F[l].preMu);
    if (rc) return rc;
    if ((rc = launch_zero_count(c, l, 3, c->F[l].preMu, S_ZEROS + l))) return rc;
    if ((rc = launch_invert(c, l, 3, c->F[l].preMu))) return rc;
  }
  return HPC_OK;
}
int pf_diags_enqueue(hpc_ctx* c, int top, double lc) {
  for (int l = 0; l <= top; ++l) {
    int rc = launch_pf_diag(c, l, lc, c->F[l].preMd);
    if (rc) return rc;
    if ((rc = launch_zero_count(c, l, 1, c->F[l].preMd, S_ZEROS + l))) return rc;
    if ((rc = launch_invert(c, l, 1, c->F[l].preMd))) return rc;
  }
  return HPC_OK;
}
int mech_diags(hpc_ctx* c, int top, double small_k) {
  const int rc = mech_diags_enqueue(c, top, small_k);
  return rc ? rc : check_zero_diags(c, top, "PreM_u");
}
int pf_diags(hpc_ctx* c, int top, double lc) {
  const int rc = pf_diags_enqueue(c, top, lc);
  return rc ? rc : check_zero_diags(c, top, "Precondition_M");
}

// pcg_u (mechanical_pcg.cpp:223-330) with preMu of level l already built.  Device scalars only.
static int pcg_u_dev(hpc_ctx* c, int l, double small_k, double Ut, int nb, int t) {
  if (nb > kMaxRelax) return arg_fail("nb_relax too large");
  if (c->fused_coarsest && l == 0) {
    const int mode = slab_coarsest_mode(c);
    if (mode == 1) return slab_coarsest(c, Ut, nb);
    if (mode == 0 && coarse_pcg_fits(c, l)) return launch_coarse_pcg(c, l, Ut, nb);
  }
  LevelFields& F = c->F[l];
  int rc;
  if ((rc = launch_bc(c, l, F.u, nullptr, 0, Ut))) return rc;  // Dirichlet_BD
  MechCall m{};
  m.level = l;
  m.finest = is_finest(c, l);
  m.epi = EPI_RESIDUAL;
  m.src = F.u;
  m.out = F.ru;
  m.small_k = small_k;
  m.fu = F.fu;
  m.set_fnorm = (t == 0 && m.finest);
  m.invM = F.preMu;
  m.s_out0 = m.set_fnorm ? S_FNORM : -1;
  m.s_out1 = slot_rz(0);
  m.s_out2 = S_RNORM;
  if ((rc = launch_mech(c, m))) return rc;
  for (int it = 0; it < nb; ++it) {
    if ((rc = launch_dir_update(c, l, 3, F.ru, F.preMu, F.p, it == 0, slot_rz(it), slot_rz(it - 1)))) return rc;
    MechCall q{};
    q.level = l;
    q.finest = m.finest;
    q.epi = EPI_PCG;
    q.src = F.p;
    q.out = F.w;
    q.small_k = small_k;
    q.s_out0 = slot_pw(it);
    q.s_out1 = q.s_out2 = -1;
    if ((rc = launch_mech(c, q))) return rc;
    if ((rc = launch_mech_update(c, l, F.p, slot_rz(it), slot_pw(it), slot_rz(it + 1), slot_rn(it)))) return rc;
  }
  return HPC_OK;
}

// pcg_d (phase_field_pcg.cpp:133-214) with preMd built; fd_norm rewritten (S_FDNORM).
static int pcg_d_dev(hpc_ctx* c, int l, double lc, int nb) {
  if (nb > kMaxRelax) return arg_fail("nb_relax too large");
  LevelFields& F = c->F[l];
  int rc;
  PfCall m{};
  m.level = l;
  m.epi = EPI_RESIDUAL;
  m.src = F.d;
  m.out = F.R;
  m.lc = lc;
  m.fd = F.fd;
  m.invM = F.preMd;
  m.s_out0 = S_FDNORM;
  m.s_out1 = S_RNORM;
  m.s_out2 = slot_rz(0);
  if ((rc = launch_pf(c, m))) return rc;
  for (int it = 0; it < nb; ++it) {
    if ((rc = launch_dir_update(c, l, 1, F.R, F.preMd, F.pd, it == 0, slot_rz(it), slot_rz(it - 1)))) return rc;
    PfCall q{};
    q.level = l;
    q.epi = EPI_PCG;
    q.src = F.pd;
    q.out = F.wd;
    q.lc = lc;
    q.s_out0 = slot_pw(it);
    q.s_out1 = q.s_out2 = -1;
    if ((rc = launch_pf(c, q))) return rc;
    if ((rc = launch_pf_update(c, l, F.pd, slot_rz(it), slot_pw(it), slot_rz(it + 1), slot_rn(it)))) return rc;
  }
  return HPC_OK;
}

static int cycle_u_dev(hpc_ctx* c, int l, const hpc_mg& mg, double small_k, double Ut, int t, long long* iters);
static int cycle_d_dev(hpc_ctx* c, int l, const hpc_mg& mg, double lc, long long* iters);

// The part of cycle_u(l) between its pre- and post-smoothing: coarsen_u, coarsen_fu, gamma cycles on
// level l-1, refine_u (mechanical_multigrid.cpp:38-48).  Below the finest level t plays no role.
static int coarse_part_u(hpc_ctx* c, int l, const hpc_mg& mg, double small_k, double Ut, int t, long long* iters) {
  int rc;
  if ((rc = launch_inject_u(c, l, Ut))) return rc;  // coarsen_u
  MechCall f{};                                      // coarsen_fu: fu_c = K_c u_c + FW(ru_f)
  f.level = l - 1;
  f.finest = false;
  f.epi = EPI_FAS;
  f.src = c->F[l - 1].u;
  f.out = c->F[l - 1].fu;
  f.small_k = small_k;
  f.rf = c->F[l].ru;
  f.fine_level = l;
  f.s_out0 = f.s_out1 = f.s_out2 = -1;
  if ((rc = launch_mech(c, f))) return rc;
  for (int j = 1; j <= mg.gamma; ++j)
    if ((rc = cycle_u_dev(c, l - 1, mg, small_k, Ut, t, iters))) return rc;
  return launch_prolong(c, l, c->F[l - 1].u, c->F[l - 1].uold, c->F[l].u, 3, true, Ut);  // refine_u
}

// cycle_u (mechanical_multigrid.cpp:18-54); returns smoother iterations via *iters.
static int cycle_u_dev(hpc_ctx* c, int l, const hpc_mg& mg, double small_k, double Ut, int t, long long* iters) {
  int rc;
  if (l == 0) {
    *iters += mg.nu0;
    return pcg_u_dev(c, 0, small_k, Ut, mg.nu0, t);
  }
  if ((rc = pcg_u_dev(c, l, small_k, Ut, mg.nu1, t))) return rc;
  *iters += mg.nu1;
  if ((rc = coarse_part_u(c, l, mg, small_k, Ut, t, iters))) return rc;
  *iters += mg.nu2;
  return pcg_u_dev(c, l, small_k, Ut, mg.nu2, t);
}

// The part of cycle_d(l) between its pre- and post-smoothing (phase_field_multigrid.cpp:39-43).
static int coarse_part_d(hpc_ctx* c, int l, const hpc_mg& mg, double lc, long long* iters) {
  int rc;
  if ((rc = launch_inject_d(c, l))) return rc;  // coarsen_d
  PfCall f{};                                    // coarsen_f_d
  f.level = l - 1;
  f.epi = EPI_FAS;
  f.src = c->F[l - 1].d;
  f.out = c->F[l - 1].fd;
  f.lc = lc;
  f.rf = c->F[l].R;
  f.fine_level = l;
  f.s_out0 = f.s_out1 = f.s_out2 = -1;
  if ((rc = launch_pf(c, f))) return rc;
  for (int j = 1; j <= mg.gamma; ++j)
    if ((rc = cycle_d_dev(c, l - 1, mg, lc, iters))) return rc;
  return launch_prolong(c, l, c->F[l - 1].d, c->F[l - 1].dold, c->F[l].d, 1, false, 0.0);  // refine_d
}

// cycle_d (phase_field_multigrid.cpp:18-44), including the nu2 x nu2 post-smoothing (:41-42).
static int cycle_d_dev(hpc_ctx* c, int l, const hpc_mg& mg, double lc, long long* iters) {
  int rc;
  if (l == 0) {
    *iters += mg.nu0;
    return pcg_d_dev(c, 0, lc, mg.nu0);
  }
  if ((rc = pcg_d_dev(c, l, lc, mg.nu1))) return rc;
  *iters += mg.nu1;
  if ((rc = coarse_part_d(c, l, mg, lc, iters))) return rc;
  for (int i = 1; i <= mg.nu2; ++i) {
    if ((rc = pcg_d_dev(c, l, lc, mg.nu2))) return rc;
    *iters += mg.nu2;
  }
  return HPC_OK;
}

// ---------------------------------------------------------------- graph replay of coarse parts
static bool same_mg(const hpc_mg& a, const hpc_mg& b) {
  return a.nu0 == b.nu0 && a.nu1 == b.nu1 && a.nu2 == b.nu2 && a.gamma == b.gamma;
}

// Runs `body` (a coarse part) through a cached CUDA graph: captured on the first call whose
// parameters differ from the cached ones (the kernels' first use must already have happened,
// `allow_capture`), replayed afterwards.  Kernel launches are counted per replay.  A graph is keyed
// by its parameters and by `flags`, the context's kernel choices baked into its launches.
static int graph_flags(const hpc_ctx* c) {
  return c->autotune * 16 + c->tma_stage * 8 + c->tc_apply * 4 + c->fused_coarsest * 2 + c->gpm_active;
}
template <class Body>
static int run_graphed(hpc_ctx* c, hpc_ctx::CoarseGraph& g, const hpc_mg& mg, double a, double b, bool allow_capture,
                       Body body, int flags) {
  const bool hit = g.valid && same_mg(g.mg, mg) && g.a == a && g.b == b && g.flags == flags;
  if (!c->use_graphs || (!hit && !allow_capture)) return body();
  if (!hit) {
    if (g.valid) {
      cudaGraphExecDestroy(g.exec);
      g.valid = 0;
    }
    HPC_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const long long k0 = c->launches;
    const int rc = body();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate");
    g.kernels = c->launches - k0;
    c->launches = k0;
    g.valid = 1;
    g.mg = mg;
    g.a = a;
    g.b = b;
    g.flags = flags;
  }
  HPC_CUDA(cudaGraphLaunch(g.exec, c->stream));
  c->launches += g.kernels;
  return HPC_OK;
}

// Top-level cycles of the solves: the finest level's smoothing is launched directly (its kernels
// are large and individually timed), everything below it is replayed as one graph.
int cycle_u_top(hpc_ctx* c, const hpc_mg& mg, double small_k, double Ut, int t, bool allow_capture) {
  const int L = c->maxlevel;
  long long it = 0;
  if (L == 0) return cycle_u_dev(c, 0, mg, small_k, Ut, t, &it);
  int rc;
  if ((rc = pcg_u_dev(c, L, small_k, Ut, mg.nu1, t))) return rc;
  if ((rc = run_graphed(c, c->gmech, mg, small_k, Ut, allow_capture,
                        [&] { return coarse_part_u(c, L, mg, small_k, Ut, t, &it); }, graph_flags(c))))
    return rc;
  return pcg_u_dev(c, L, small_k, Ut, mg.nu2, t);
}

int cycle_d_top(hpc_ctx* c, const hpc_mg& mg, double lc, bool allow_capture) {
  const int L = c->maxlevel;
  long long it = 0;
  if (L == 0) return cycle_d_dev(c, 0, mg, lc, &it);
  int rc;
  if ((rc = pcg_d_dev(c, L, lc, mg.nu1))) return rc;
  if ((rc = run_graphed(c, c->gpf, mg, lc, 0.0, allow_capture, [&] { return coarse_part_d(c, L, mg, lc, &it); },
                        graph_flags(c))))
    return rc;
  for (int i = 1; i <= mg.nu2; ++i)
    if ((rc = pcg_d_dev(c, L, lc, mg.nu2))) return rc;
  return HPC_OK;
}

// Per-level element moduli for the mechanical solve: MP_choice + MP_all_element on the finest level,
// then VR_all_level for K_element and G_element (mechanical_displacement.cpp:33-45).
int mech_material(hpc_ctx* c, double small_k) {
  int rc;
  const int L = c->maxlevel;
  if ((rc = launch_choice_level(c, L, small_k, true, true))) return rc;
  for (int l = L; l > 0; --l) {
    if ((rc = launch_vr(c, l, c->F[l].Ke, c->F[l - 1].Ke, true, true))) return rc;
    if ((rc = launch_vr(c, l, c->F[l].Ge, c->F[l - 1].Ge, true, true))) return rc;
  }
  return HPC_OK;
}

// Gauss-point moduli of the finest level for the solve about to run; while the returned scope lives,
// the finest applies read them (the material does not change during a mechanical solve).
struct GpmScope {
  hpc_ctx* c;
  explicit GpmScope(hpc_ctx* ctx) : c(ctx) {}
  ~GpmScope() { c->gpm_active = 0; }
};
int gp_material(hpc_ctx* c, double small_k) {
  LevelFields& F = c->F[c->maxlevel];
  if (!F.gpm) {
    const size_t bytes = sizeof(double) * 16 * (size_t)c->L[c->maxlevel].n;
    HPC_CUDA(ctx_alloc(c, (void**)&F.gpm, bytes));
    HPC_CUDA(cudaMemsetAsync(F.gpm, 0, bytes, c->stream));  // non-element slots stay zero
  }
  int rc = launch_gp_material(c, small_k);
  if (rc) return rc;
  c->gpm_active = 1;
  return HPC_OK;
}

// Kernels whose bounded waits ran out (tensor-core applies, TMA staging) report it in S_ERR.
int check_wait_error(hpc_ctx* c) {
  double err = 0.0;
  int rc;
  if ((rc = read_scalars(c, S_ERR, 1, &err))) return rc;
  if (err != 0.0) {
    write_scalar(c, S_ERR, 0.0);
    set_error("a bounded wait in a kernel (tensor copy or MMA completion) ran out");
    return HPC_ERR_CUDA;
  }
  return HPC_OK;
}

// u_entire (mechanical_displacement.cpp:25-115).
static int u_entire_dev(hpc_ctx* c, const hpc_mg& mg, double small_k, double Ut, int t, double mech_tol, int* cycles,
                        long long* fin_iters) {
  int rc;
  const int L = c->maxlevel;
  if ((rc = write_scalar(c, S_FNORM, c->f_norm))) return rc;
  if ((rc = mech_material(c, small_k))) return rc;
  if ((rc = mech_diags(c, L, small_k))) return rc;
  GpmScope gpm_scope(c);
  if (L > 0 && (rc = gp_material(c, small_k))) return rc;
  // Initial_residual_u (mechanical_pcg.cpp:193-220): no Dirichlet_BD on u, no reaction copy
  MechCall m{};
  m.level = L;
  m.finest = true;
  m.epi = EPI_RESIDUAL;
  m.src = c->F[L].u;
  m.out = c->F[L].ru;
  m.small_k = small_k;
  m.fu = c->F[L].fu;
  m.set_fnorm = false;
  m.invM = nullptr;
  m.s_out0 = m.s_out1 = -1;
  m.s_out2 = S_RNORM;
  if ((rc = launch_mech(c, m))) return rc;
  double s3[3];
  if ((rc = read_scalars(c, S_FNORM, 3, s3))) return rc;
  double r_norm = s3[S_RNORM], f_norm = s3[S_FNORM];
  double rel = 1.0;
  if (t >= 1 && f_norm != 0) rel = r_norm / f_norm;
  *cycles = 0;
  *fin_iters = 0;
  const int per_cycle = (L == 0) ? mg.nu0 : mg.nu1 + mg.nu2;
  for (int j = 1; j <= mg.ncy; ++j) {
    if (rel > mech_tol) {
      if ((rc = cycle_u_top(c, mg, small_k, Ut, t, *cycles > 0))) return rc;
      ++*cycles;
      *fin_iters += per_cycle;
      if ((rc = launch_dot(c, L, 3, c->F[L].ru, nullptr, S_RNORM))) return rc;
      if ((rc = read_scalars(c, S_FNORM, 3, s3))) return rc;
      r_norm = s3[S_RNORM];
      f_norm = s3[S_FNORM];
      rel = r_norm / f_norm;
    }
    if (rel <= mech_tol) break;
  }
  if (c->tma_stage && (rc = check_wait_error(c))) return rc;
  c->f_norm = f_norm;
  // externe_force_nodal (mechanical_right_hnd.cpp:18-38)
  if ((rc = launch_bc(c, L, c->F[L].u, nullptr, 0, Ut))) return rc;
  MechCall r{};
  r.level = L;
  r.finest = true;
  r.epi = EPI_REACTION;
  r.src = c->F[L].u;
  r.out = c->F[L].fu;
  r.small_k = small_k;
  r.s_out0 = r.s_out1 = r.s_out2 = -1;
  return launch_mech(c, r);
}

// ---------------------------------------------------------------- precision form: FP32 V-cycle
// The preconditioner of the mixed-precision solve: one V-cycle of cycle_u's kind (restarted
// Jacobi-PCG smoothing, injection, FAS right-hand side, prolongation) on single-precision copies of
// the levels, solving for a correction (homogeneous Dirichlet values).  Its coarsest solve stays FP64.
int ensure_f32(hpc_ctx* c) {
  if (c->F32[0].u) return HPC_OK;
  for (int l = 0; l <= c->maxlevel; ++l) {
    const size_t n = (size_t)c->L[l].n;
    LevelF32& F = c->F32[l];
    float** vec[] = {&F.u, &F.fu, &F.ru, &F.uold, &F.p, &F.w, &F.invM};
    for (float** p : vec) {
      HPC_CUDA(ctx_alloc(c, (void**)p, 3 * n * sizeof(float)));
      HPC_CUDA(cudaMemsetAsync(*p, 0, 3 * n * sizeof(float), c->stream));
    }
    float** mat_f[] = {&F.K, &F.G, &F.d};
    float** mat_c[] = {&F.Ke, &F.Ge};
    const bool fin = (l == c->maxlevel);
    if (fin && l > 0) {
      HPC_CUDA(ctx_alloc(c, (void**)&F.gpm, 16 * n * sizeof(float)));
      HPC_CUDA(cudaMemsetAsync(F.gpm, 0, 16 * n * sizeof(float), c->stream));
    }
    for (int q = 0; q < (fin ? 3 : 2); ++q) {
      float** p = fin ? mat_f[q] : mat_c[q];
      HPC_CUDA(ctx_alloc(c, (void**)p, n * sizeof(float)));
      HPC_CUDA(cudaMemsetAsync(*p, 0, n * sizeof(float), c->stream));
    }
  }
  return HPC_OK;
}

// FP32 material and inverse diagonals from the FP64 ones (after mech_material and mech_diags).
int f32_material(hpc_ctx* c) {
  int rc;
  for (int l = 0; l <= c->maxlevel; ++l) {
    const long long n = c->L[l].n;
    LevelF32& G = c->F32[l];
    const LevelFields& F = c->F[l];
    if ((rc = launch_to_f32(c, F.preMu, G.invM, 3 * n))) return rc;
    if (l == c->maxlevel) {
      if ((rc = launch_to_f32(c, F.bulK, G.K, n))) return rc;
      if ((rc = launch_to_f32(c, F.G, G.G, n))) return rc;
      if ((rc = launch_to_f32(c, F.d, G.d, n))) return rc;
      if (c->gpm_active && G.gpm && (rc = launch_to_f32(c, F.gpm, G.gpm, 16 * n))) return rc;
    } else {
      if ((rc = launch_to_f32(c, F.Ke, G.Ke, n))) return rc;
      if ((rc = launch_to_f32(c, F.Ge, G.Ge, n))) return rc;
    }
  }
  return HPC_OK;
}

// pcg_u (mechanical_pcg.cpp:223-330) on the FP32 mirror, homogeneous Dirichlet values.
// u_zero: the unknown is known to be zero (the finest pre-smoother of the correction), so the first
// residual is f itself and needs no operator apply.
static int pcg_u32(hpc_ctx* c, int l, double small_k, int nb, bool u_zero = false) {
  if (nb > kMaxRelax) return arg_fail("nb_relax too large");
  LevelF32& F = c->F32[l];
  int rc;
  MechCall32 m{};
  m.level = l;
  m.finest = is_finest(c, l);
  if (u_zero) {
    if ((rc = launch_residual_zero_f32(c, l, slot_rz(0)))) return rc;
  } else {
    if ((rc = launch_bc_zero_f32(c, l, F.u))) return rc;
    m.epi = EPI_RESIDUAL;
    m.src = F.u;
    m.out = F.ru;
    m.small_k = small_k;
    m.fu = F.fu;
    m.invM = F.invM;
    m.s_out0 = -1;
    m.s_out1 = slot_rz(0);
    m.s_out2 = -1;
    if ((rc = launch_mech_f32(c, m))) return rc;
  }
  for (int it = 0; it < nb; ++it) {
    if ((rc = launch_dir_update_f32(c, l, it == 0, slot_rz(it), slot_rz(it - 1)))) return rc;
    MechCall32 q{};
    q.level = l;
    q.finest = m.finest;
    q.epi = EPI_PCG;
    q.src = F.p;
    q.out = F.w;
    q.small_k = small_k;
    q.s_out0 = slot_pw(it);
    q.s_out1 = q.s_out2 = -1;
    if ((rc = launch_mech_f32(c, q))) return rc;
    if ((rc = launch_mech_update_f32(c, l, slot_rz(it), slot_pw(it), slot_rz(it + 1), slot_rn(it)))) return rc;
  }
  return HPC_OK;
}

// The coarsest level in FP64: pcg_u with nu0 iterations on the FP64 arrays of level 0.
static int coarsest64(hpc_ctx* c, const hpc_mg& mg, double small_k) {
  const long long n3 = 3 * c->L[0].n;
  int rc;
  if ((rc = launch_to_f64(c, c->F32[0].u, c->F[0].u, n3))) return rc;
  if ((rc = launch_to_f64(c, c->F32[0].fu, c->F[0].fu, n3))) return rc;
  if ((rc = pcg_u_dev(c, 0, small_k, 0.0, mg.nu0, 1))) return rc;
  return launch_to_f32(c, c->F[0].u, c->F32[0].u, n3);
}

static int cycle_u32(hpc_ctx* c, int l, const hpc_mg& mg, double small_k);

static int coarse_part_u32(hpc_ctx* c, int l, const hpc_mg& mg, double small_k) {
  int rc;
  if ((rc = launch_inject_u_f32(c, l))) return rc;
  MechCall32 f{};
  f.level = l - 1;
  f.finest = false;
  f.epi = EPI_FAS;
  f.src = c->F32[l - 1].u;
  f.out = c->F32[l - 1].fu;
  f.small_k = small_k;
  f.rf = c->F32[l].ru;
  f.fine_level = l;
  f.s_out0 = f.s_out1 = f.s_out2 = -1;
  if ((rc = launch_mech_f32(c, f))) return rc;
  for (int j = 1; j <= mg.gamma; ++j)
    if ((rc = cycle_u32(c, l - 1, mg, small_k))) return rc;
  return launch_prolong_f32(c, l);
}

static int cycle_u32(hpc_ctx* c, int l, const hpc_mg& mg, double small_k) {
  int rc;
  if (l == 0) return coarsest64(c, mg, small_k);
  if ((rc = pcg_u32(c, l, small_k, mg.nu1))) return rc;
  if ((rc = coarse_part_u32(c, l, mg, small_k))) return rc;
  return pcg_u32(c, l, small_k, mg.nu2);
}

// ---------------------------------------------------------------- flexible PCG (precision form)
int ensure_fcg(hpc_ctx* c) {
  if (c->fcg.x) return HPC_OK;
  const size_t bytes = sizeof(double) * 3 * (size_t)c->L[c->maxlevel].n;
  double** arrs[] = {&c->fcg.x, &c->fcg.r, &c->fcg.rp, &c->fcg.f, &c->fcg.p};
  for (double** a : arrs) {
    HPC_CUDA(ctx_alloc(c, (void**)a, bytes));
    HPC_CUDA(cudaMemsetAsync(*a, 0, bytes, c->stream));
  }
  return HPC_OK;
}

// True residual r = f - K x with Dirichlet rows zero; at t == 0 the reactions of x become f's
// Dirichlet rows and f_norm (as every finest pcg_u call at t == 0 does, mechanical_pcg.cpp:252-258).
int fcg_residual(hpc_ctx* c, double small_k, int t, int s_rn) {
  const int L = c->maxlevel;
  MechCall m{};
  m.level = L;
  m.finest = true;
  m.epi = EPI_RESIDUAL;
  m.src = c->fcg.x;
  m.out = c->fcg.r;
  m.small_k = small_k;
  m.fu = c->fcg.f;
  m.set_fnorm = (t == 0);
  m.invM = nullptr;
  m.s_out0 = m.set_fnorm ? S_FNORM : -1;
  m.s_out1 = -1;
  m.s_out2 = s_rn;
  return launch_mech(c, m);
}

// One flexible-PCG iteration k of the mechanical solve (the part without a host read): the
// preconditioning V-cycle (FP32 mirror when mixed), delta / gamma, the direction, w = K p and the
// x / r update.  coarse_graph: replay the cycle's coarse part from its cached graph.
int fcg_iteration(hpc_ctx* c, const hpc_mg& mg, double small_k, int k, bool mixed, bool coarse_graph) {
  const int L = c->maxlevel;
  LevelFields& F = c->F[L];
  const LevelGeo& g = c->L[L];
  const size_t vbytes = sizeof(double) * 3 * (size_t)g.n;
  int r2;
  // z = V-cycle on A z = r from z = 0 with homogeneous Dirichlet values: u is the cycle's unknown,
  // fu its right-hand side
  if (mixed) {  // the same cycle on the FP32 mirror; z comes back to F.u in FP64
    const LevelF32& G = c->F32[L];
    HPC_CUDA(cudaMemsetAsync(G.u, 0, 3 * (size_t)g.n * sizeof(float), c->stream));
    if ((r2 = launch_to_f32(c, c->fcg.r, G.fu, 3 * g.n))) return r2;
    if (L == 0) {
      if ((r2 = cycle_u32(c, 0, mg, small_k))) return r2;
    } else {
      if ((r2 = pcg_u32(c, L, small_k, mg.nu1, true))) return r2;
      if (coarse_graph) {
        if ((r2 = run_graphed(c, c->g32, mg, small_k, 0.0, k > 0, [&] { return coarse_part_u32(c, L, mg, small_k); },
                              graph_flags(c))))
          return r2;
      } else if ((r2 = coarse_part_u32(c, L, mg, small_k))) {
        return r2;
      }
      if ((r2 = pcg_u32(c, L, small_k, mg.nu2))) return r2;
    }
  } else {
    HPC_CUDA(cudaMemsetAsync(F.u, 0, vbytes, c->stream));
    HPC_CUDA(cudaMemcpyAsync(F.fu, c->fcg.r, vbytes, cudaMemcpyDeviceToDevice, c->stream));
    if ((r2 = cycle_u_top(c, mg, small_k, 0.0, 1, k > 0))) return r2;
  }
  // delta_k = (z, r_k), gamma_k = (z, r_{k-1}); p = z + beta p.  The precision form reads z from the
  // FP32 cycle directly (its FP64 copy would be exact).
  if (mixed) {
    const float* z = c->F32[L].u;
    if ((r2 = launch_dot2(c, L, z, c->fcg.r, k > 0 ? c->fcg.rp : nullptr, slot_fdelta(k), slot_fgamma(k))))
      return r2;
    if ((r2 = launch_fcg_dir(c, L, z, c->fcg.p, k == 0, slot_fdelta(k), slot_fgamma(k), slot_fdelta(k - 1))))
      return r2;
  } else {
    if ((r2 = launch_dot2(c, L, F.u, c->fcg.r, k > 0 ? c->fcg.rp : nullptr, slot_fdelta(k), slot_fgamma(k))))
      return r2;
    if ((r2 = launch_fcg_dir(c, L, F.u, c->fcg.p, k == 0, slot_fdelta(k), slot_fgamma(k), slot_fdelta(k - 1))))
      return r2;
  }
  // w = K p, (p, w); the smoothers' own p and w are free between V-cycles
  MechCall q{};
  q.level = L;
  q.finest = true;
  q.epi = EPI_PCG;
  q.src = c->fcg.p;
  q.out = F.w;
  q.small_k = small_k;
  q.s_out0 = slot_fpw(k);
  q.s_out1 = q.s_out2 = -1;
  if ((r2 = launch_mech(c, q))) return r2;
  // r_{k-1} kept for the flexible beta; x += alpha p, r -= alpha w, alpha = delta_k / (p, w)
  HPC_CUDA(cudaMemcpyAsync(c->fcg.rp, c->fcg.r, vbytes, cudaMemcpyDeviceToDevice, c->stream));
  return launch_mech_update_on(c, L, c->fcg.x, c->fcg.r, c->fcg.p, F.w, F.preMu, slot_fdelta(k), slot_fpw(k),
                               slot_fdummy(k), slot_frn(k));
}

// The mechanical solve of u_entire (mechanical_displacement.cpp:25-115) by flexible PCG on the finest
// level, preconditioned by one multigrid V-cycle of the reference's kind (FAS with restarted
// Jacobi-PCG smoothers, which on the linear correction problem acts as a correction-scheme cycle).
// The outer iteration keeps the true residual, the dot products and the x / r / p updates in FP64;
// the stopping test is the reference's |r|^2 / |f|^2 <= mech_tol.  *cycles = V-cycles (one per
// iteration), *fin_iters = finest smoother iterations inside them.
static int u_entire_fcg_dev(hpc_ctx* c, const hpc_mg& mg, double small_k, double Ut, int t, double mech_tol,
                            int* cycles, long long* fin_iters, bool mixed) {
  int rc;
  const int L = c->maxlevel;
  LevelFields& F = c->F[L];
  const LevelGeo& g = c->L[L];
  const size_t vbytes = sizeof(double) * 3 * (size_t)g.n;
  if ((rc = ensure_fcg(c))) return rc;
  if (mg.ncy + 1 > kMaxRelax) return arg_fail("ncy too large");
  if ((rc = write_scalar(c, S_FNORM, c->f_norm))) return rc;
  if ((rc = mech_material(c, small_k))) return rc;
  if ((rc = mech_diags(c, L, small_k))) return rc;
  GpmScope gpm_scope(c);
  if (L > 0 && (rc = gp_material(c, small_k))) return rc;
  if (mixed) {
    if ((rc = ensure_f32(c))) return rc;
    if ((rc = f32_material(c))) return rc;
  }
  // x = u with the Dirichlet values, f = fu (saved: the V-cycle uses fu as its right-hand side)
  if ((rc = launch_bc(c, L, F.u, nullptr, 0, Ut))) return rc;
  HPC_CUDA(cudaMemcpyAsync(c->fcg.x, F.u, vbytes, cudaMemcpyDeviceToDevice, c->stream));
  HPC_CUDA(cudaMemcpyAsync(c->fcg.f, F.fu, vbytes, cudaMemcpyDeviceToDevice, c->stream));
  if ((rc = fcg_residual(c, small_k, t, slot_frn(-1)))) return rc;
  double s2[2];
  if ((rc = read_scalars(c, S_FNORM, 1, s2))) return rc;
  if ((rc = read_scalars(c, slot_frn(-1), 1, s2 + 1))) return rc;
  double f_norm = s2[0], rel = f_norm != 0 ? s2[1] / f_norm : 1.0;
  *cycles = 0;
  *fin_iters = 0;
  const int per_cycle = (L == 0) ? mg.nu0 : mg.nu1 + mg.nu2;
  // The precision form's iteration has no host read until its residual norm: with graphs on (and no
  // launch timing), each iteration of one class (k = 0, odd k, even k) is captured once and replayed.
  const bool whole_graph = mixed && c->use_graphs && c->timing_class < 0;
  for (int k = 0; k < mg.ncy; ++k) {
    if (rel <= mech_tol && !(t == 0 && k == 0)) break;  // one iteration forced at t == 0 (:74, :84-85)
    auto iteration = [&](bool coarse_graph) -> int { return fcg_iteration(c, mg, small_k, k, mixed, coarse_graph); };
    if (whole_graph) {
      // graph key: the cycle parameters, small_k and the kernel choices baked into the launches
      hpc_ctx::CoarseGraph& gk = c->gfcg[k == 0 ? 0 : ((k & 1) ? 1 : 2)];
      if ((rc = run_graphed(c, gk, mg, small_k, 0.0, true, [&] { return iteration(false); }, graph_flags(c)))) return rc;
    } else if ((rc = iteration(true))) {
      return rc;
    }
    ++*cycles;
    *fin_iters += per_cycle;
    // The stopping decision is always taken on the true residual f - K x: at t == 0 it is computed
    // every iteration (f_norm follows the reactions of the current iterate); later the recursive
    // residual is used until it passes the test, then the true one confirms it or replaces it.
    double rn;
    if (t == 0) {
      if ((rc = fcg_residual(c, small_k, t, slot_frn(k)))) return rc;
      if ((rc = read_scalars(c, S_FNORM, 1, &f_norm))) return rc;
      if ((rc = read_scalars(c, slot_frn(k), 1, &rn))) return rc;
    } else {
      if ((rc = read_scalars(c, slot_frn(k), 1, &rn))) return rc;
      if (f_norm != 0 && rn / f_norm <= mech_tol) {
        if ((rc = fcg_residual(c, small_k, t, slot_frn(k)))) return rc;
        if ((rc = read_scalars(c, slot_frn(k), 1, &rn))) return rc;
      }
    }
    rel = f_norm != 0 ? rn / f_norm : 1.0;
  }
  if (((mixed && c->tc_apply) || c->tma_stage) && (rc = check_wait_error(c))) return rc;
  c->f_norm = f_norm;
  // u = x, fu restored; externe_force_nodal (mechanical_right_hnd.cpp:18-38)
  HPC_CUDA(cudaMemcpyAsync(F.u, c->fcg.x, vbytes, cudaMemcpyDeviceToDevice, c->stream));
  HPC_CUDA(cudaMemcpyAsync(F.fu, c->fcg.f, vbytes, cudaMemcpyDeviceToDevice, c->stream));
  if ((rc = launch_bc(c, L, F.u, nullptr, 0, Ut))) return rc;
  MechCall r{};
  r.level = L;
  r.finest = true;
  r.epi = EPI_REACTION;
  r.src = F.u;
  r.out = F.fu;
  r.small_k = small_k;
  r.s_out0 = r.s_out1 = r.s_out2 = -1;
  return launch_mech(c, r);
}

// phase_field (phase_field.cpp:15-57).
static int phase_field_dev(hpc_ctx* c, const hpc_mg& mg, double lc, double pf_tol, int* cycles, long long* fin_iters) {
  int rc;
  const int L = c->maxlevel;
  if ((rc = write_scalar(c, S_FDNORM, c->fd_norm))) return rc;
  if ((rc = pf_diags(c, L, lc))) return rc;
  PfCall m{};  // initial_residual (phase_field_pcg.cpp:106-131)
  m.level = L;
  m.epi = EPI_RESIDUAL;
  m.src = c->F[L].d;
  m.out = c->F[L].R;
  m.lc = lc;
  m.fd = c->F[L].fd;
  m.s_out0 = -1;
  m.s_out1 = S_RNORM;
  m.s_out2 = -1;
  if ((rc = launch_pf(c, m))) return rc;
  double s3[3];
  if ((rc = read_scalars(c, S_FNORM, 3, s3))) return rc;
  double r_norm = s3[S_RNORM], fd_norm = s3[S_FDNORM];
  double sres = 1.0;
  *cycles = 0;
  *fin_iters = 0;
  const int per_cycle = (L == 0) ? mg.nu0 : mg.nu1 + mg.nu2 * mg.nu2;
  for (int j = 1; j <= mg.ncy; ++j) {
    if (r_norm > pf_tol) {
      if (sres > pf_tol) {
        if ((rc = cycle_d_top(c, mg, lc, *cycles > 0))) return rc;
        ++*cycles;
        *fin_iters += per_cycle;
      }
      if ((rc = launch_dot(c, L, 1, c->F[L].R, nullptr, S_RNORM))) return rc;
      if ((rc = read_scalars(c, S_FNORM, 3, s3))) return rc;
      r_norm = s3[S_RNORM];
      fd_norm = s3[S_FDNORM];
      sres = r_norm / fd_norm;
      if (sres <= pf_tol) break;
    } else {
      break;
    }
  }
  c->fd_norm = fd_norm;
  return HPC_OK;
}

int voigt_all_level(hpc_ctx* c, int field) {
  int rc;
  for (int l = c->maxlevel; l > 0; --l)
    if ((rc = launch_vr(c, l, scalar_field(c, field, l), scalar_field(c, field, l - 1), false, false))) return rc;
  return HPC_OK;
}

}  // namespace hpc

using namespace hpc;

// =============================================================================================
// C ABI
// =============================================================================================
extern "C" {

const char* hpc_last_error(void) { return g_err.c_str(); }

static int footprint(const hpc_geometry* geo, int nr, int r, size_t* bytes) {
  if (!geometry_ok(geo, nr, r) || !bytes) return arg_fail("bad geometry");
  double box[6];
  HostLevel lv[kMaxLevels];
  host_geometry(*geo, box, lv);
  SlabLevel sl[kMaxLevels];
  slab_levels(*geo, nr, r, sl);
  const int nz0 = lv[0].nz;  // the whole coarsest level (a split gathers it)
  for (int l = 0; l <= geo->maxlevel; ++l) lv[l].nz = sl[l].nz;
  size_t total = 0;
  if (nr > 1) total += sizeof(double) * 14 * (size_t)lv[0].px * lv[0].ny * nz0 + nz0;
  for (int l = 0; l <= geo->maxlevel; ++l) {
    long long n = (long long)lv[l].px * lv[l].ny * lv[l].nz;
    total += level_bytes(n) + (size_t)(lv[l].nx + lv[l].ny + lv[l].nz);
  }
  const HostLevel& f = lv[geo->maxlevel];
  const size_t nf = (size_t)f.px * f.ny * f.nz;
  total += nf * sizeof(double);  // d_old
  total += sizeof(double) * (kScalarPool + 3 * 8192) + 64;
  // allocated on first use: Gauss-point moduli (16 n), flexible-PCG vectors (5 x 3n), the FP32
  // mirror of every level (7 x 3n + material) with its Gauss-point moduli, the checkpoint (6 dense)
  total += nf * sizeof(double) * (16 + 15);
  for (int l = 0; l <= geo->maxlevel; ++l) {
    const size_t n = (size_t)lv[l].px * lv[l].ny * lv[l].nz;
    total += n * sizeof(float) * (21 + (l == geo->maxlevel ? 3 + 16 : 2));
  }
  total += 6 * (size_t)f.nx * f.ny * f.nz * sizeof(double);
  total += (size_t)f.nx * f.ny * f.nz * sizeof(double);  // upload staging
  *bytes = total;
  return HPC_OK;
}

int hpc_footprint(const hpc_geometry* geo, size_t* bytes) { return footprint(geo, 1, 0, bytes); }

int hpc_footprint_slab(const hpc_geometry* geo, int nranks, int rank, size_t* bytes) {
  if (nranks < 1 || rank < 0 || rank >= nranks) return arg_fail("bad slab rank");
  return footprint(geo, nranks, rank, bytes);
}

static std::atomic<unsigned long long> g_ctx_uid{0};

// hpc_create (a whole specimen) and hpc_create_slab (rank r of nr along z; `slab`).
static int create_ctx(hpc_ctx** out, const hpc_geometry* geo, int device, int nr, int r, bool slab) {
  if (!out) return arg_fail("null output");
  *out = nullptr;
  if (!geometry_ok(geo, nr, r)) return arg_fail("bad geometry");
  SlabLevel sl[kMaxLevels];
  if (!slab_levels(*geo, nr, r, sl)) return arg_fail("bad slab decomposition (every rank needs a coarsest plane)");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_error("no CUDA device: the library has no CPU path");
    return HPC_ERR_NODEVICE;
  }
  if (device < 0 || device >= ndev) return arg_fail("bad device index");
  HPC_CUDA(cudaSetDevice(device));
  pool_setup(device);
  hpc_ctx* c = new hpc_ctx();
  std::memset(c, 0, sizeof(*c));
  c->geo = *geo;
  c->maxlevel = geo->maxlevel;
  c->device = device;
  c->choice_quirk = 1;
  c->use_graphs = 1;
  c->uid = ++g_ctx_uid;
  c->fused_coarsest = 1;
  c->tma_stage = 1;  // tensor-copy staging of the finest applies: the same bits, 3 % faster on 257^3
  c->timing_class = HPC_KC_NONE;
  HostLevel lv[kMaxLevels];
  host_geometry(*geo, c->box, lv);
  for (int l = 0; l <= c->maxlevel; ++l) lv[l].nz = sl[l].nz;  // this rank's planes (all of them for one rank)
  auto fail = [&](int rc) {
    hpc_destroy(c);
    return rc;
  };
  if (slab) {
    // no graph replay of coarse parts until the slab joins NCCL (hpc_slab_join_nccl): the in-process
    // transport waits on the host inside them; the coarsest level is gathered and solved redundantly
    c->use_graphs = 0;
    const int rc = slab_attach(c, nr, r);
    if (rc) return fail(rc);
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "stream"));
  // axis flags for the Dirichlet sets (boundary_conditions.cpp:20-68, coordinates as get_coordinate :14-18)
  size_t flag_bytes = 0;
  for (int l = 0; l <= c->maxlevel; ++l) flag_bytes += lv[l].nx + lv[l].ny + lv[l].nz;
  std::vector<uint8_t> hflags(flag_bytes);
  {
    cudaError_t ae = ctx_alloc(c, &c->bc_dev_base, flag_bytes);
    if (ae != cudaSuccess) return fail(cuda_fail(ae, "cudaMallocAsync(flags)"));
  }
  size_t off = 0;
  const double* B = c->box;
  for (int l = 0; l <= c->maxlevel; ++l) {
    const HostLevel& h = lv[l];
    LevelGeo& g = c->L[l];
    g.nx = h.nx;
    g.ny = h.ny;
    g.nz = h.nz;
    g.px = h.px;
    g.plane = (long long)h.px * h.ny;
    g.n = g.plane * h.nz;
    g.hx = h.hx;
    g.hy = h.hy;
    g.hz = h.hz;
    g.wg = 0.125 * h.hx * h.hy * h.hz;
    g.zb = sl[l].zb;
    g.oz0 = sl[l].lo;
    g.oz1 = sl[l].hi;
    g.zsh = l < c->maxlevel ? 2 * sl[l].zb - sl[l + 1].zb : 0;
    if (g.zsh != 0 && g.zsh != -1) return fail(arg_fail("slab levels do not nest"));
    uint8_t* fx = hflags.data() + off;
    uint8_t* fy = fx + h.nx;
    uint8_t* fz = fy + h.ny;
    for (int i = 0; i < h.nx; ++i) {
      const double x = B[0] + i * h.hx;
      fx[i] = (uint8_t)((x == 0.5 * (B[0] + B[1]) ? 1 : 0) | (x == B[1] ? 2 : 0));
    }
    for (int j = 0; j < h.ny; ++j) {
      const double y = B[2] + j * h.hy;
      fy[j] = (uint8_t)((y == B[2] ? 1 : 0) | (y == 0.5 * (B[2] + B[3]) ? 2 : 0));
    }
    for (int k = 0; k < h.nz; ++k) {
      const double z = B[4] + (sl[l].zb + k) * h.hz;
      fz[k] = (uint8_t)((z == B[4] ? 1 : 0) | (z == B[5] ? 2 : 0));
    }
    uint8_t* dbase = (uint8_t*)c->bc_dev_base + off;
    g.bx = dbase;
    g.by = dbase + h.nx;
    g.bz = dbase + h.nx + h.ny;
    off += h.nx + h.ny + h.nz;
  }
  if (cudaMemcpyAsync(c->bc_dev_base, hflags.data(), flag_bytes, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    return fail(cuda_fail(cudaGetLastError(), "flags upload"));
  // per-level arrays
  for (int l = 0; l <= c->maxlevel; ++l) {
    const long long n = c->L[l].n;
    LevelFields& F = c->F[l];
    double** scal[] = {&F.bulK, &F.G, &F.gc, &F.d, &F.H, &F.fd, &F.Ke, &F.Ge, &F.R, &F.dold, &F.preMd, &F.pd, &F.wd, &F.tmp1};
    double** vec[] = {&F.u, &F.fu, &F.ru, &F.uold, &F.preMu, &F.p, &F.w, &F.tmp3};
    for (double** p : scal) {
      cudaError_t ae = ctx_alloc(c, (void**)p, sizeof(double) * n);
      if (ae != cudaSuccess) return fail(cuda_fail(ae, "cudaMallocAsync(level field)"));
      if (cudaMemsetAsync(*p, 0, sizeof(double) * n, c->stream) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "memset"));
    }
    for (double** p : vec) {
      cudaError_t ae = ctx_alloc(c, (void**)p, sizeof(double) * 3 * n);
      if (ae != cudaSuccess) return fail(cuda_fail(ae, "cudaMallocAsync(level vector)"));
      if (cudaMemsetAsync(*p, 0, sizeof(double) * 3 * n, c->stream) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "memset"));
    }
    cudaError_t ae = ctx_alloc(c, (void**)&F.choice, (size_t)n);
    if (ae != cudaSuccess) return fail(cuda_fail(ae, "cudaMallocAsync(choice)"));
    if (cudaMemsetAsync(F.choice, 0, (size_t)n, c->stream) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "memset"));
  }
  {
    const long long n = c->L[c->maxlevel].n;
    cudaError_t ae = ctx_alloc(c, (void**)&c->d_old, sizeof(double) * n);
    if (ae != cudaSuccess) return fail(cuda_fail(ae, "cudaMallocAsync(d_old)"));
    cudaMemsetAsync(c->d_old, 0, sizeof(double) * n, c->stream);
    c->partials_cap = 3 * 8192;
    if ((ae = ctx_alloc(c, (void**)&c->scal, sizeof(double) * kScalarPool)) != cudaSuccess) return fail(cuda_fail(ae, "scal"));
    cudaMemsetAsync(c->scal, 0, sizeof(double) * kScalarPool, c->stream);
    if ((ae = ctx_alloc(c, (void**)&c->partials, sizeof(double) * c->partials_cap)) != cudaSuccess)
      return fail(cuda_fail(ae, "partials"));
    if ((ae = ctx_alloc(c, (void**)&c->counter, sizeof(unsigned int) * 4)) != cudaSuccess) return fail(cuda_fail(ae, "counter"));
    cudaMemsetAsync(c->counter, 0, sizeof(unsigned int) * 4, c->stream);
    if (!(c->hscal = pinned_slot())) return fail(cuda_fail(cudaErrorMemoryAllocation, "pinned"));
  }
  double N[64];
  shape_table(N);
  int rc = upload_shape_table(N);
  if (rc) return fail(rc);
  if ((rc = coarse_pcg_prepare())) return fail(rc);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "create sync"));
  *out = c;
  return HPC_OK;
}

int hpc_create(hpc_ctx** out, const hpc_geometry* geo, int device) {
  return create_ctx(out, geo, device, 1, 0, false);
}

int hpc_create_slab(hpc_ctx** out, const hpc_geometry* geo, int device, int nranks, int rank) {
  if (nranks < 1 || rank < 0 || rank >= nranks) return arg_fail("bad slab rank");
  return create_ctx(out, geo, device, nranks, rank, true);
}

int hpc_destroy(hpc_ctx* c) {
  if (!c) return HPC_OK;
  cudaSetDevice(c->device);
  vtk_release(c);
  // graphs first: a slab's may hold NCCL calls of the communicator slab_release destroys
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->gmech.valid) cudaGraphExecDestroy(c->gmech.exec);
  if (c->gpf.valid) cudaGraphExecDestroy(c->gpf.exec);
  if (c->g32.valid) cudaGraphExecDestroy(c->g32.exec);
  for (auto& gf : c->gfcg)
    if (gf.valid) cudaGraphExecDestroy(gf.exec);
  c->gmech.valid = c->gpf.valid = c->g32.valid = 0;
  for (auto& gf : c->gfcg) gf.valid = 0;
  slab_release(c);
  for (int l = 0; l <= c->maxlevel && l < kMaxLevels; ++l) {
    LevelFields& F = c->F[l];
    void* ptrs[] = {F.bulK, F.G, F.gc, F.d, F.H, F.fd, F.Ke, F.Ge, F.R, F.dold, F.preMd, F.pd, F.wd, F.tmp1,
                    F.u, F.fu, F.ru, F.uold, F.preMu, F.p, F.w, F.tmp3, F.choice, F.gpm};
    for (void* p : ptrs) ctx_free(c, p);
  }
  ctx_free(c, c->d_old);
  ctx_free(c, c->scal);
  ctx_free(c, c->partials);
  ctx_free(c, c->counter);
  ctx_free(c, c->bc_dev_base);
  ctx_free(c, c->stage);
  {
    double* fa[] = {c->fcg.x, c->fcg.r, c->fcg.rp, c->fcg.f, c->fcg.p};
    for (double* p : fa) ctx_free(c, p);
  }
  for (int l = 0; l <= c->maxlevel && l < kMaxLevels; ++l) {
    LevelF32& G = c->F32[l];
    float* fa[] = {G.u, G.fu, G.ru, G.uold, G.p, G.w, G.invM, G.K, G.G, G.d, G.Ke, G.Ge, G.gpm};
    for (float* p : fa) ctx_free(c, p);
  }
  if (c->stream) cudaStreamSynchronize(c->stream);  // every release in the pool before the stream goes
  pinned_release(c->hscal);
  for (int i = 0; i < 2 * c->tev_cap; ++i) cudaEventDestroy(c->tev[i]);
  delete[] c->tev;
  if (c->ck.stream) cudaStreamSynchronize(c->ck.stream);
  if (c->ck.dev) cudaFree(c->ck.dev);
  if (c->ck.host) cudaFreeHost(c->ck.host);
  if (c->ck.snap) cudaEventDestroy(c->ck.snap);
  if (c->ck.done) cudaEventDestroy(c->ck.done);
  if (c->ck.stream) cudaStreamDestroy(c->ck.stream);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return HPC_OK;
}

int hpc_level_dims(hpc_ctx* c, int level, int* n3, double* h3) {
  if (!c || level < 0 || level > c->maxlevel) return arg_fail("bad level");
  const LevelGeo& g = c->L[level];
  if (n3) { n3[0] = g.nx; n3[1] = g.ny; n3[2] = g.nz; }
  if (h3) { h3[0] = g.hx; h3[1] = g.hy; h3[2] = g.hz; }
  return HPC_OK;
}

int hpc_sync(hpc_ctx* c) {
  if (!c) return arg_fail("null context");
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  return HPC_OK;
}

int hpc_set_tensor_apply(hpc_ctx* c, int on) {
  if (!c) return arg_fail("null context");
  c->tc_apply = on != 0;
  return HPC_OK;
}

int hpc_set_fused_coarsest(hpc_ctx* c, int on) {
  if (!c) return arg_fail("null context");
  c->fused_coarsest = on != 0;
  return HPC_OK;
}

int hpc_set_tma_staging(hpc_ctx* c, int on) {
  if (!c) return arg_fail("null context");
  c->tma_stage = on != 0;
  return HPC_OK;
}

int hpc_set_autotune(hpc_ctx* c, int on) {
  if (!c) return arg_fail("null context");
  // trial launches differ between ranks, and every reducing launch of a slab is a collective step
  if (c->slab && on) return arg_fail("no strip autotuning on a slab");
  c->autotune = on != 0;
  return HPC_OK;
}

int hpc_tuned_shapes(int* out5, int cap, int* count) {
  if (!count || (cap > 0 && !out5)) return arg_fail("bad argument");
  *count = tuned_shapes(out5, cap);
  return HPC_OK;
}

int hpc_set_choice_quirk(hpc_ctx* c, int reproduce) {
  if (!c) return arg_fail("null context");
  c->choice_quirk = reproduce != 0;
  return HPC_OK;
}

int hpc_launch_count(hpc_ctx* c, long long* count, int reset) {
  if (!c) return arg_fail("null context");
  if (count) *count = c->launches;
  if (reset) c->launches = 0;
  return HPC_OK;
}

void* hpc_stream(hpc_ctx* c) { return c ? (void*)c->stream : nullptr; }

int hpc_binary_version(int* version) {
  if (!version) return arg_fail("null pointer");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device: the library has no CPU path");
    return HPC_ERR_NODEVICE;
  }
  HPC_CUDA(kernel_binary_version(version));
  return HPC_OK;
}

int hpc_kernel_timing(hpc_ctx* c, int kernel_class) {
  if (!c) return arg_fail("null context");
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  c->timing_class = kernel_class;
  c->tev_used = 0;
  return HPC_OK;
}

int hpc_kernel_time(hpc_ctx* c, long long* launches, double* total_ms) {
  if (!c) return arg_fail("null context");
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  double tot = 0.0;
  for (int i = 0; i < c->tev_used; ++i) {
    float ms = 0.f;
    HPC_CUDA(cudaEventElapsedTime(&ms, c->tev[2 * i], c->tev[2 * i + 1]));
    tot += ms;
  }
  if (launches) *launches = c->tev_used;
  if (total_ms) *total_ms = tot;
  return HPC_OK;
}

// A dense x-fastest host array into the pitched device array d of a level, asynchronously on the
// context's stream: one contiguous copy into a dense device buffer and an unpack kernel (a pitched
// host-to-device copy of short rows runs at a fraction of the link's bandwidth).  The host array
// must stay valid until the stream has passed the copy.
static int upload_dense(hpc_ctx* c, int level, double* d, const double* host) {
  if (!c->stage) {
    const LevelGeo& f = c->L[c->maxlevel];
    HPC_CUDA(ctx_alloc(c, (void**)&c->stage, sizeof(double) * (size_t)f.nx * f.ny * f.nz));
  }
  const LevelGeo& g = c->L[level];
  HPC_CUDA(cudaMemcpyAsync(c->stage, host, sizeof(double) * (size_t)g.nx * g.ny * g.nz, cudaMemcpyHostToDevice,
                           c->stream));
  return launch_unpack(c, level, c->stage, d);
}

int hpc_upload(hpc_ctx* c, int field, int level, int comp, const double* host) {
  if (!c || !host) return arg_fail("null argument");
  double* d = component(c, field, level, comp);
  if (!d) return arg_fail("bad field/level/component");
  HPC_CUDA(cudaSetDevice(c->device));
  if (const int rc = upload_dense(c, level, d, host)) return rc;
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  return HPC_OK;
}

int hpc_download(hpc_ctx* c, int field, int level, int comp, double* host) {
  if (!c || !host) return arg_fail("null argument");
  double* d = component(c, field, level, comp);
  if (!d) return arg_fail("bad field/level/component");
  const LevelGeo& g = c->L[level];
  HPC_CUDA(cudaSetDevice(c->device));
  HPC_CUDA(cudaMemcpy2DAsync(host, sizeof(double) * g.nx, d, sizeof(double) * g.px, sizeof(double) * g.nx,
                             (size_t)g.ny * g.nz, cudaMemcpyDeviceToHost, c->stream));
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  return HPC_OK;
}

int hpc_upload_choice(hpc_ctx* c, int level, const int16_t* host) {
  if (!c || !host || level < 0 || level > c->maxlevel) return arg_fail("bad argument");
  const LevelGeo& g = c->L[level];
  std::vector<int8_t> tmp((size_t)g.n, 0);
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i)
        tmp[(size_t)i + (size_t)j * g.px + (size_t)k * g.plane] =
            (int8_t)host[(size_t)i + (size_t)j * g.nx + (size_t)k * g.nx * g.ny];
  HPC_CUDA(cudaMemcpyAsync(c->F[level].choice, tmp.data(), (size_t)g.n, cudaMemcpyHostToDevice, c->stream));
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  return HPC_OK;
}

int hpc_download_choice(hpc_ctx* c, int level, int16_t* host) {
  if (!c || !host || level < 0 || level > c->maxlevel) return arg_fail("bad argument");
  const LevelGeo& g = c->L[level];
  std::vector<int8_t> tmp((size_t)g.n);
  HPC_CUDA(cudaMemcpyAsync(tmp.data(), c->F[level].choice, (size_t)g.n, cudaMemcpyDeviceToHost, c->stream));
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < g.nz; ++k)
    for (int j = 0; j < g.ny; ++j)
      for (int i = 0; i < g.nx; ++i)
        host[(size_t)i + (size_t)j * g.nx + (size_t)k * g.nx * g.ny] = tmp[(size_t)i + (size_t)j * g.px + (size_t)k * g.plane];
  return HPC_OK;
}

int hpc_get_state(hpc_ctx* c, double* s6) {
  if (!c || !s6) return arg_fail("null argument");
  s6[0] = c->f_norm; s6[1] = c->fd_norm; s6[2] = c->Ue; s6[3] = c->Ut; s6[4] = c->dU; s6[5] = c->uprop;
  return HPC_OK;
}
int hpc_set_state(hpc_ctx* c, const double* s6) {
  if (!c || !s6) return arg_fail("null argument");
  c->f_norm = s6[0]; c->fd_norm = s6[1]; c->Ue = s6[2]; c->Ut = s6[3]; c->dU = s6[4]; c->uprop = s6[5];
  return HPC_OK;
}

// ---------------------------------------------------------------- checkpoint / restart
// The staggered loop's whole state between two increments is the finest u (3 components), H, d,
// d_old and the six loop scalars: every coarse field, the regimes and the right-hand sides are
// rebuilt from them by the next increment (crack_propagation.cpp:65-121).
static double* ck_source(hpc_ctx* c, int i) {
  const int L = c->maxlevel;
  switch (i) {
    case 0: case 1: case 2: return c->F[L].u + (long long)i * c->L[L].n;
    case 3: return c->F[L].H;
    case 4: return c->F[L].d;
    default: return c->d_old;
  }
}

int hpc_checkpoint_begin(hpc_ctx* c, int t) {
  if (!c) return arg_fail("null context");
  HPC_CUDA(cudaSetDevice(c->device));
  const LevelGeo& g = c->L[c->maxlevel];
  const size_t dense = (size_t)g.nx * g.ny * g.nz;
  hpc_ctx::Checkpoint& k = c->ck;
  if (!k.dev) {  // first checkpoint of this context: buffers, copy stream and events
    HPC_CUDA(cudaMalloc((void**)&k.dev, 6 * dense * sizeof(double)));
    HPC_CUDA(cudaMallocHost((void**)&k.host, 6 * dense * sizeof(double)));
    HPC_CUDA(cudaStreamCreateWithFlags(&k.stream, cudaStreamNonBlocking));
    HPC_CUDA(cudaEventCreateWithFlags(&k.snap, cudaEventDisableTiming));
    HPC_CUDA(cudaEventCreateWithFlags(&k.done, cudaEventDisableTiming));
  }
  // the previous copy must have left the snapshot before it is overwritten
  if (k.pending) HPC_CUDA(cudaStreamWaitEvent(c->stream, k.done, 0));
  for (int i = 0; i < 6; ++i)
    HPC_CUDA(cudaMemcpy2DAsync(k.dev + i * dense, sizeof(double) * g.nx, ck_source(c, i), sizeof(double) * g.px,
                               sizeof(double) * g.nx, (size_t)g.ny * g.nz, cudaMemcpyDeviceToDevice, c->stream));
  HPC_CUDA(cudaEventRecord(k.snap, c->stream));
  HPC_CUDA(cudaStreamWaitEvent(k.stream, k.snap, 0));
  HPC_CUDA(cudaMemcpyAsync(k.host, k.dev, 6 * dense * sizeof(double), cudaMemcpyDeviceToHost, k.stream));
  HPC_CUDA(cudaEventRecord(k.done, k.stream));
  k.t = t;
  k.pending = 1;
  k.valid = 1;
  k.state[0] = c->f_norm; k.state[1] = c->fd_norm; k.state[2] = c->Ue;
  k.state[3] = c->Ut; k.state[4] = c->dU; k.state[5] = c->uprop;
  return HPC_OK;
}

int hpc_checkpoint_wait(hpc_ctx* c, int* t, const double** fields, double* state6) {
  if (!c) return arg_fail("null context");
  hpc_ctx::Checkpoint& k = c->ck;
  if (!k.valid) return arg_fail("no checkpoint has been started");
  HPC_CUDA(cudaSetDevice(c->device));
  if (k.pending) {
    HPC_CUDA(cudaEventSynchronize(k.done));
    k.pending = 0;
  }
  if (t) *t = k.t;
  if (fields) *fields = k.host;
  if (state6)
    for (int i = 0; i < 6; ++i) state6[i] = k.state[i];
  return HPC_OK;
}

int hpc_checkpoint_restore(hpc_ctx* c, const double* u, const double* v, const double* w, const double* H,
                           const double* d, const double* d_old, const double* state6) {
  if (!c || !u || !v || !w || !H || !d || !d_old || !state6) return arg_fail("null argument");
  HPC_CUDA(cudaSetDevice(c->device));
  const double* src[6] = {u, v, w, H, d, d_old};
  for (int i = 0; i < 6; ++i)
    if (const int rc = upload_dense(c, c->maxlevel, ck_source(c, i), src[i])) return rc;
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  return hpc_set_state(c, state6);
}

// ---------------------------------------------------------------- operators
int hpc_internal_force(hpc_ctx* c, int level, int src_field, int dst_field, double small_k) {
  if (!c) return arg_fail("null context");
  double* s = vector_field(c, src_field, level);
  double* d = vector_field(c, dst_field, level);
  if (!s || !d || s == d) return arg_fail("bad fields");
  MechCall m{};
  m.level = level;
  m.finest = is_finest(c, level);
  m.epi = EPI_PLAIN;
  m.src = s;
  m.out = d;
  m.small_k = small_k;
  m.s_out0 = m.s_out1 = m.s_out2 = -1;
  int rc = launch_mech(c, m);
  return rc ? rc : hpc_sync(c);
}

int hpc_prem_u(hpc_ctx* c, int level, int dst_field, double small_k) {
  if (!c) return arg_fail("null context");
  double* d = vector_field(c, dst_field, level);
  if (!d) return arg_fail("bad field");
  int rc = launch_mech_diag(c, level, is_finest(c, level), small_k, d);
  return rc ? rc : hpc_sync(c);
}

int hpc_fld(hpc_ctx* c, int level, int src_field, int dst_field, double lc) {
  if (!c) return arg_fail("null context");
  double* s = scalar_field(c, src_field, level);
  double* d = scalar_field(c, dst_field, level);
  if (!s || !d || s == d) return arg_fail("bad fields");
  PfCall p{};
  p.level = level;
  p.epi = EPI_PLAIN;
  p.src = s;
  p.out = d;
  p.lc = lc;
  p.s_out0 = p.s_out1 = p.s_out2 = -1;
  int rc = launch_pf(c, p);
  return rc ? rc : hpc_sync(c);
}

int hpc_precondition_m(hpc_ctx* c, int level, int dst_field, double lc) {
  if (!c) return arg_fail("null context");
  double* d = scalar_field(c, dst_field, level);
  if (!d) return arg_fail("bad field");
  int rc = launch_pf_diag(c, level, lc, d);
  return rc ? rc : hpc_sync(c);
}

// ---------------------------------------------------------------- smoothers and solves
int hpc_initial_residual_u(hpc_ctx* c, int level, double small_k, double* r_norm) {
  if (!c || level < 0 || level > c->maxlevel) return arg_fail("bad argument");
  MechCall m{};
  m.level = level;
  m.finest = is_finest(c, level);
  m.epi = EPI_RESIDUAL;
  m.src = c->F[level].u;
  m.out = c->F[level].ru;
  m.small_k = small_k;
  m.fu = c->F[level].fu;
  m.s_out0 = m.s_out1 = -1;
  m.s_out2 = S_RNORM;
  int rc = launch_mech(c, m);
  if (rc) return rc;
  double s3[3];
  if ((rc = read_scalars(c, 0, 3, s3))) return rc;
  if (r_norm) *r_norm = s3[S_RNORM];
  return HPC_OK;
}

int hpc_pcg_u(hpc_ctx* c, int level, double small_k, double Ut, int nb_relax, int t, double* f_norm) {
  if (!c || level < 0 || level > c->maxlevel || nb_relax < 0 || !f_norm) return arg_fail("bad argument");
  int rc;
  if ((rc = write_scalar(c, S_FNORM, *f_norm))) return rc;
  if ((rc = launch_mech_diag(c, level, is_finest(c, level), small_k, c->F[level].preMu))) return rc;
  if ((rc = launch_zero_count(c, level, 3, c->F[level].preMu, S_ZEROS))) return rc;
  if (nb_relax > 0 && (rc = check_zero_diags(c, 0, "PreM_u"))) return rc;
  if ((rc = launch_invert(c, level, 3, c->F[level].preMu))) return rc;
  if ((rc = pcg_u_dev(c, level, small_k, Ut, nb_relax, t))) return rc;
  if ((rc = read_scalars(c, S_FNORM, 1, f_norm))) return rc;
  return HPC_OK;
}

int hpc_initial_residual_d(hpc_ctx* c, int level, double lc, double* r_norm) {
  if (!c || level < 0 || level > c->maxlevel) return arg_fail("bad argument");
  PfCall m{};
  m.level = level;
  m.epi = EPI_RESIDUAL;
  m.src = c->F[level].d;
  m.out = c->F[level].R;
  m.lc = lc;
  m.fd = c->F[level].fd;
  m.s_out0 = -1;
  m.s_out1 = S_RNORM;
  m.s_out2 = -1;
  int rc = launch_pf(c, m);
  if (rc) return rc;
  double s3[3];
  if ((rc = read_scalars(c, 0, 3, s3))) return rc;
  if (r_norm) *r_norm = s3[S_RNORM];
  return HPC_OK;
}

int hpc_pcg_d(hpc_ctx* c, int level, double lc, int nb_relax, int t, double* fd_norm) {
  (void)t;
  if (!c || level < 0 || level > c->maxlevel || nb_relax < 0 || !fd_norm) return arg_fail("bad argument");
  int rc;
  if ((rc = launch_pf_diag(c, level, lc, c->F[level].preMd))) return rc;
  if ((rc = launch_zero_count(c, level, 1, c->F[level].preMd, S_ZEROS))) return rc;
  if (nb_relax > 0 && (rc = check_zero_diags(c, 0, "Precondition_M"))) return rc;
  if ((rc = launch_invert(c, level, 1, c->F[level].preMd))) return rc;
  if ((rc = pcg_d_dev(c, level, lc, nb_relax))) return rc;
  return read_scalars(c, S_FDNORM, 1, fd_norm);
}

int hpc_cycle_u(hpc_ctx* c, int level, const hpc_mg* mg, double small_k, double Ut, int t, double* f_norm) {
  if (!c || !mg || level < 0 || level > c->maxlevel || !f_norm) return arg_fail("bad argument");
  int rc;
  if ((rc = write_scalar(c, S_FNORM, *f_norm))) return rc;
  if ((rc = mech_diags(c, level, small_k))) return rc;
  long long it = 0;
  if ((rc = cycle_u_dev(c, level, *mg, small_k, Ut, t, &it))) return rc;
  return read_scalars(c, S_FNORM, 1, f_norm);
}

int hpc_cycle_d(hpc_ctx* c, int level, const hpc_mg* mg, double lc, int t, double* fd_norm) {
  (void)t;
  if (!c || !mg || level < 0 || level > c->maxlevel || !fd_norm) return arg_fail("bad argument");
  int rc;
  if ((rc = write_scalar(c, S_FDNORM, *fd_norm))) return rc;
  if ((rc = pf_diags(c, level, lc))) return rc;
  long long it = 0;
  if ((rc = cycle_d_dev(c, level, *mg, lc, &it))) return rc;
  return read_scalars(c, S_FDNORM, 1, fd_norm);
}

int hpc_u_entire(hpc_ctx* c, const hpc_mg* mg, double small_k, double Ut, int t, double* f_norm, double mech_tol,
                 int* cycles, int* iters) {
  if (!c || !mg || !f_norm) return arg_fail("bad argument");
  c->f_norm = *f_norm;
  int cy = 0;
  long long it = 0;
  int rc = u_entire_dev(c, *mg, small_k, Ut, t, mech_tol, &cy, &it);
  if (rc) return rc;
  if ((rc = hpc_sync(c))) return rc;
  *f_norm = c->f_norm;
  if (cycles) *cycles = cy;
  if (iters) *iters = (int)it;
  return HPC_OK;
}

int hpc_u_entire_fcg(hpc_ctx* c, const hpc_mg* mg, double small_k, double Ut, int t, double* f_norm,
                     double mech_tol, int mixed, int* cycles, int* iters) {
  if (!c || !mg || !f_norm) return arg_fail("bad argument");
  c->f_norm = *f_norm;
  int cy = 0;
  long long it = 0;
  int rc = u_entire_fcg_dev(c, *mg, small_k, Ut, t, mech_tol, &cy, &it, mixed != 0);
  if (rc) return rc;
  if ((rc = hpc_sync(c))) return rc;
  *f_norm = c->f_norm;
  if (cycles) *cycles = cy;
  if (iters) *iters = (int)it;
  return HPC_OK;
}

int hpc_phase_field(hpc_ctx* c, const hpc_mg* mg, double lc, int t, double* fd_norm, double pf_tol, int* cycles,
                    int* iters) {
  (void)t;
  if (!c || !mg || !fd_norm) return arg_fail("bad argument");
  c->fd_norm = *fd_norm;
  int cy = 0;
  long long it = 0;
  int rc = phase_field_dev(c, *mg, lc, pf_tol, &cy, &it);
  if (rc) return rc;
  *fd_norm = c->fd_norm;
  if (cycles) *cycles = cy;
  if (iters) *iters = (int)it;
  return HPC_OK;
}

}  // extern "C"

namespace hpc {

// The part of an increment between the two solves (crack_propagation.cpp:71-85): the load schedule
// at t == 0, the history update, its Voigt averages and the phase-field right-hand sides.
int step_mid(hpc_ctx* c, const hpc_step_params* p) {
  const double U_unit = 1.0;
  const int L = c->maxlevel;
  int rc;
  if (p->t == 0) {
    if (p->ut0 <= 0.0) {
      double ue;
      if ((rc = launch_ue(c, p->lc, S_RES0))) return rc;
      if ((rc = read_scalars(c, S_RES0, 1, &ue))) return rc;
      c->Ue = ue;
      c->Ut = ue;
      c->dU = p->du_factor * ue;
    } else {
      c->Ue = p->ut0;
      c->Ut = p->ut0;
      c->dU = p->du;
    }
    c->uprop = c->Ut / U_unit;
  }
  if ((rc = launch_strain_history(c, p->lc, c->uprop))) return rc;
  if ((rc = voigt_all_level(c, HPC_H))) return rc;
  for (int l = L; l >= 0; --l)
    if ((rc = launch_fd_h(c, l))) return rc;
  return HPC_OK;
}

// The end of an increment (crack_propagation.cpp:86-121): d maxima with the d_old update, the top
// reaction sum, the next load, the step outputs.
int step_end_enqueue(hpc_ctx* c) {
  int rc;
  if ((rc = launch_dmax(c, S_RES0, S_RES1, true))) return rc;
  return launch_top_sum(c, S_RES2);
}
int step_end(hpc_ctx* c, const hpc_step_params* p, int mcy, long long mit, int pcy, long long pit, double* out) {
  const int rc = step_end_enqueue(c);
  return rc ? rc : step_end_finish(c, p, mcy, mit, pcy, pit, out);
}
int step_end_finish(hpc_ctx* c, const hpc_step_params* p, int mcy, long long mit, int pcy, long long pit, double* out) {
  const double U_unit = 1.0;
  int rc;
  double r3[4];  // d maxima, top sum, and S_ERR: a bounded wait of a kernel in this increment ran out
  if ((rc = read_scalars(c, S_RES0, 4, r3))) return rc;
  if (r3[3] != 0.0) {
    write_scalar(c, S_ERR, 0.0);
    set_error("a bounded wait in a kernel (tensor copy or MMA completion) ran out");
    return HPC_ERR_CUDA;
  }
  const double FeW = r3[2] * p->voxel_size;
  const double Ut_now = c->Ut;
  c->Ut = c->Ut + c->dU;
  c->uprop = c->Ut / U_unit;
  out[0] = Ut_now;
  out[1] = c->uprop * FeW;
  out[2] = r3[0];
  out[3] = r3[1];
  out[4] = mcy;
  out[5] = pcy;
  out[6] = (double)mit;
  out[7] = (double)pit;
  return HPC_OK;
}

}  // namespace hpc

extern "C" {

int hpc_step(hpc_ctx* c, const hpc_step_params* p, double* out) {
  if (!c || !p || !out) return arg_fail("bad argument");
  const double U_unit = 1.0;
  int rc, mcy = 0, pcy = 0;
  long long mit = 0, pit = 0;
  if (p->mech_solver == HPC_MECH_FCG || p->mech_solver == HPC_MECH_MIXED) {
    if ((rc = u_entire_fcg_dev(c, p->mg_u, p->small_k, U_unit, p->t, p->mech_tol, &mcy, &mit,
                               p->mech_solver == HPC_MECH_MIXED)))
      return rc;
  } else if (p->mech_solver == HPC_MECH_FAS) {
    if ((rc = u_entire_dev(c, p->mg_u, p->small_k, U_unit, p->t, p->mech_tol, &mcy, &mit))) return rc;
  } else {
    return arg_fail("unknown mech_solver");
  }
  if ((rc = step_mid(c, p))) return rc;
  if ((rc = phase_field_dev(c, p->mg_d, p->lc, p->pf_tol, &pcy, &pit))) return rc;
  return step_end(c, p, mcy, mit, pcy, pit, out);
}

// ---------------------------------------------------------------- material / history
int hpc_mp_choice(hpc_ctx* c) {
  if (!c) return arg_fail("null context");
  int rc;
  for (int l = c->maxlevel; l >= 0; --l)
    if ((rc = launch_mp_choice_level(c, l))) return rc;
  return hpc_sync(c);
}
int hpc_mp_all_element(hpc_ctx* c, double small_k) {
  if (!c) return arg_fail("null context");
  int rc = launch_choice_level(c, c->maxlevel, small_k, false, true);
  return rc ? rc : hpc_sync(c);
}
int hpc_vr_all_level(hpc_ctx* c, int field) {
  if (!c || !scalar_field(c, field, 0)) return arg_fail("bad field");
  int rc;
  for (int l = c->maxlevel; l > 0; --l)
    if ((rc = launch_vr(c, l, scalar_field(c, field, l), scalar_field(c, field, l - 1), true, true))) return rc;
  return hpc_sync(c);
}
int hpc_voigt_all_level(hpc_ctx* c, int field) {
  if (!c || !scalar_field(c, field, 0)) return arg_fail("bad field");
  int rc = voigt_all_level(c, field);
  return rc ? rc : hpc_sync(c);
}
int hpc_coarse_vr(hpc_ctx* c, int field) {
  if (!c || !scalar_field(c, field, 0)) return arg_fail("bad field");
  int rc;
  for (int l = c->maxlevel; l > 0; --l)
    if ((rc = launch_coarse_vr(c, l, scalar_field(c, field, l), scalar_field(c, field, l - 1)))) return rc;
  return hpc_sync(c);
}
int hpc_strain_history(hpc_ctx* c, double lc, double u_proportion) {
  if (!c) return arg_fail("null context");
  int rc = launch_strain_history(c, lc, u_proportion);
  return rc ? rc : hpc_sync(c);
}
int hpc_fd_h(hpc_ctx* c, int level) {
  if (!c || level < 0 || level > c->maxlevel) return arg_fail("bad level");
  int rc = launch_fd_h(c, level);
  return rc ? rc : hpc_sync(c);
}
int hpc_delta_d_max(hpc_ctx* c, double* out) {
  if (!c || !out) return arg_fail("bad argument");
  int rc = launch_dmax(c, S_RES0, S_RES1, false);
  return rc ? rc : read_scalars(c, S_RES0, 1, out);
}
int hpc_d_max(hpc_ctx* c, double* out) {
  if (!c || !out) return arg_fail("bad argument");
  int rc = launch_dmax(c, S_RES0, S_RES1, false);
  return rc ? rc : read_scalars(c, S_RES1, 1, out);
}
int hpc_U_e(hpc_ctx* c, double lc, double* out) {
  if (!c || !out) return arg_fail("bad argument");
  int rc = launch_ue(c, lc, S_RES0);
  return rc ? rc : read_scalars(c, S_RES0, 1, out);
}
int hpc_externe_force_nodal(hpc_ctx* c, double Ut, double small_k) {
  if (!c) return arg_fail("null context");
  const int L = c->maxlevel;
  int rc;
  if ((rc = launch_bc(c, L, c->F[L].u, nullptr, 0, Ut))) return rc;
  MechCall r{};
  r.level = L;
  r.finest = true;
  r.epi = EPI_REACTION;
  r.src = c->F[L].u;
  r.out = c->F[L].fu;
  r.small_k = small_k;
  r.s_out0 = r.s_out1 = r.s_out2 = -1;
  if ((rc = launch_mech(c, r))) return rc;
  return hpc_sync(c);
}
int hpc_externe_force_sum(hpc_ctx* c, double* out) {
  if (!c || !out) return arg_fail("bad argument");
  int rc = launch_top_sum(c, S_RES0);
  return rc ? rc : read_scalars(c, S_RES0, 1, out);
}
int hpc_initial_crack(hpc_ctx* c, double H_crack, int level) {
  if (!c || level < 0 || level > c->maxlevel) return arg_fail("bad level");
  const LevelGeo& g = c->L[level];
  const LevelGeo& gm = c->L[c->maxlevel];
  const double* B = c->box;
  std::vector<uint8_t> f((size_t)g.nx + g.ny + g.nz);
  for (int i = 0; i < g.nx; ++i) f[i] = (B[0] + i * g.hx) == B[1];
  for (int j = 0; j < g.ny; ++j) f[g.nx + j] = (B[2] + j * g.hy) == B[3];
  for (int k = 0; k < g.nz; ++k) {
    const double z = B[4] + (g.zb + k) * g.hz;
    f[g.nx + g.ny + k] = (z == 0.5 * (B[4] + B[5]) || z == 0.5 * (B[4] + B[5]) - gm.hz);
  }
  uint8_t* d = nullptr;
  HPC_CUDA(cudaMalloc(&d, f.size()));
  cudaMemcpy(d, f.data(), f.size(), cudaMemcpyHostToDevice);
  int rc = launch_crack(c, level, d, d + g.nx, d + g.nx + g.ny, H_crack);
  cudaStreamSynchronize(c->stream);
  cudaFree(d);
  return rc;
}

// ---------------------------------------------------------------- boundary conditions
int hpc_dirichlet_bd(hpc_ctx* c, int level, int field, double Ut) {
  if (!c) return arg_fail("null context");
  double* v = vector_field(c, field, level);
  if (!v) return arg_fail("bad field");
  int rc = launch_bc(c, level, v, nullptr, 0, Ut);
  return rc ? rc : hpc_sync(c);
}
int hpc_dirichlet_force(hpc_ctx* c, int level, int f_field, int fi_field) {
  if (!c) return arg_fail("null context");
  double* f = vector_field(c, f_field, level);
  double* fi = vector_field(c, fi_field, level);
  if (!f || !fi) return arg_fail("bad field");
  int rc = launch_bc(c, level, f, fi, 1, 0.0);
  return rc ? rc : hpc_sync(c);
}
int hpc_dirichlet_residual(hpc_ctx* c, int level, int field) {
  if (!c) return arg_fail("null context");
  double* v = vector_field(c, field, level);
  if (!v) return arg_fail("bad field");
  int rc = launch_bc(c, level, v, nullptr, 2, 0.0);
  return rc ? rc : hpc_sync(c);
}

// ---------------------------------------------------------------- transfers
int hpc_solution_injection(hpc_ctx* c, int field, int comp, int lf) {
  if (!c || lf < 1 || lf > c->maxlevel) return arg_fail("bad level");
  double* f = component(c, field, lf, comp);
  double* co = component(c, field, lf - 1, comp);
  if (!f || !co) return arg_fail("bad field");
  int rc = launch_inject(c, lf, f, co, 1);
  return rc ? rc : hpc_sync(c);
}
int hpc_coarsen_f_standard(hpc_ctx* c, int fc_field, int rf_field, int fic_field, int comp, int lf) {
  if (!c || lf < 1 || lf > c->maxlevel) return arg_fail("bad level");
  double* fc = component(c, fc_field, lf - 1, comp);
  double* rf = component(c, rf_field, lf, comp);
  double* fic = component(c, fic_field, lf - 1, comp);
  if (!fc || !rf || !fic || fc == fic) return arg_fail("bad field");
  int rc = launch_restrict(c, lf, rf, fic, fc, 1);
  return rc ? rc : hpc_sync(c);
}
int hpc_refine_standard(hpc_ctx* c, int uf_field, int uc_field, int ucold_field, int comp, int lf) {
  if (!c || lf < 1 || lf > c->maxlevel) return arg_fail("bad level");
  double* uf = component(c, uf_field, lf, comp);
  double* uc = component(c, uc_field, lf - 1, comp);
  double* uo = component(c, ucold_field, lf - 1, comp);
  if (!uf || !uc || !uo) return arg_fail("bad field");
  int rc = launch_prolong(c, lf, uc, uo, uf, 1, false, 0.0);
  return rc ? rc : hpc_sync(c);
}

// ---------------------------------------------------------------- input path
int hpc_image_material(hpc_ctx* c, const uint8_t* image, const int* voxel_n, int ngray, const int* gray,
                       const double* E, const double* nu, const double* gcv, double voxel_size) {
  if (!c || !image || !voxel_n || ngray < 2 || !gray || !E || !nu || !gcv) return arg_fail("bad argument");
  const LevelGeo& g = c->L[c->maxlevel];
  for (int a = 0; a < 3; ++a) {
    const int need = (a == 0 ? g.nx : a == 1 ? g.ny : g.zb + g.nz) + c->geo.roi_start[a];
    if (voxel_n[a] < need) {
      set_error("image smaller than the ROI of the finest grid");
      return HPC_ERR_INPUT;
    }
  }
  const size_t nvox = (size_t)voxel_n[0] * voxel_n[1] * voxel_n[2];
  uint8_t* dimg = nullptr;
  void* dtab = nullptr;
  HPC_CUDA(ctx_alloc(c, (void**)&dimg, nvox));
  const size_t tab_bytes = sizeof(int) * ngray + 3 * sizeof(double) * ngray + 64;
  if (ctx_alloc(c, &dtab, tab_bytes) != cudaSuccess) {
    ctx_free(c, dimg);
    return cuda_fail(cudaErrorMemoryAllocation, "cudaMallocAsync(table)");
  }
  double* dE = (double*)dtab;
  double* dnu = dE + ngray;
  double* dgc = dnu + ngray;
  int* dgray = (int*)(dgc + ngray);
  cudaMemcpyAsync(dimg, image, nvox, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(dE, E, sizeof(double) * ngray, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(dnu, nu, sizeof(double) * ngray, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(dgc, gcv, sizeof(double) * ngray, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(dgray, gray, sizeof(int) * ngray, cudaMemcpyHostToDevice, c->stream);
  int rc = launch_image_material(c, dimg, voxel_n, ngray, dgray, dE, dnu, dgc, voxel_size);
  ctx_free(c, dimg);
  ctx_free(c, dtab);
  if (rc) return rc;
  for (int f : {HPC_BULK, HPC_G, HPC_GC})
    for (int l = c->maxlevel; l > 0; --l)
      if ((rc = launch_coarse_vr(c, l, scalar_field(c, f, l), scalar_field(c, f, l - 1)))) return rc;
  return hpc_sync(c);
}

}  // extern "C"
