// Batched staggered increments: many specimens of uneven sizes advanced by one increment each, with
// every solve loop driven on the device.
//
// hpc_step decides after every V-cycle on the host whether to go on (one scalar read per cycle, where
// the reference tests convergence).  For a batch that is one host round trip per cycle per specimen.
// Here each specimen's mechanical solve and phase-field solve become a conditional WHILE node of a
// CUDA graph: its body is the specimen's V-cycle (or flexible-PCG iteration) followed by a one-thread
// kernel that updates the loop state in the context's scalar pool and sets the node's condition with
// the reference's stopping rule.  The graph of a batch holds one such chain per specimen, side by side
// and independent, so ONE graph launch runs every specimen's whole solve to its own convergence,
// each at its own pace: specimens of different sizes do not wait for one another between cycles.
//
// The bodies are the same launches, with the same arguments and scalar slots, as the host-driven
// solves make, so a specimen's results in a batch are bit-identical to hpc_step on it alone.
// The work around the loops (regimes, diagonals, Gauss-point moduli, history, right-hand sides,
// reductions) is enqueued per specimen on its own stream by the one calling thread.
//
// Every loop is bounded on the device: the condition is (cycles < ncy) && (not converged), with the
// cycle count incremented by every body run, so a loop ends after at most ncy bodies whatever the
// residuals are (a NaN residual fails the "not converged" comparison and ends it too).
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace hpc {
namespace {

enum LoopKind : int { LOOP_FAS = 0, LOOP_PF = 1, LOOP_FCG = 2 };

struct LoopRule {
  int kind;
  int ncy;
  int t;
  double tol;
};

// The reference's continuation tests: mechanical |r|^2/|f|^2 > tol (mechanical_displacement.cpp:
// 86-108), phase field |R|^2 > tol and |R|^2/|fd|^2 > tol (phase_field.cpp:30-43); at most ncy cycles.
__device__ __forceinline__ unsigned loop_go(const LoopRule& r, const double* s) {
  if (!(s[S_LCOUNT] < (double)r.ncy)) return 0u;
  if (r.kind == LOOP_PF) return (s[S_RNORM] > r.tol && s[S_LREL] > r.tol) ? 1u : 0u;
  return s[S_LREL] > r.tol ? 1u : 0u;
}

// Start of a solve loop: the state after the solve's initial residual, and the loop's condition.
//   FAS: rel = |r|^2/|f|^2 from t >= 1 on (1 at t == 0, where one cycle is forced);
//   PF:  sres = 1 (the first cycle runs if |R|^2 > tol);
//   FCG: rel = |r|^2/|f|^2 of the true residual; one iteration forced at t == 0.
__global__ void loop_gate_kernel(cudaGraphConditionalHandle h, double* s, LoopRule r, int s_rn0) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  s[S_LCOUNT] = 0.0;
  s[S_LTRUE] = 0.0;
  double rel = 1.0;
  if (r.kind == LOOP_FAS) {
    const double rn = s[S_RNORM], fn = s[S_FNORM];
    if (r.t >= 1 && fn != 0.0) rel = rn / fn;
  } else if (r.kind == LOOP_FCG) {
    const double rn = s[s_rn0], fn = s[S_FNORM];
    rel = fn != 0.0 ? rn / fn : 1.0;
  }
  s[S_LREL] = rel;
  unsigned go = loop_go(r, s);
  if (r.kind == LOOP_FCG && r.t == 0 && r.ncy > 0) go = 1u;
  cudaGraphSetConditional(h, go);
}

// A WHILE node's condition from the state the first (IF-gated) flexible-PCG iteration left.
__global__ void loop_rearm_kernel(cudaGraphConditionalHandle h, const double* s, LoopRule r) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  cudaGraphSetConditional(h, loop_go(r, s));
}

// End of one body run: count it, take the loop's ratio from the norms the body left, and (when the
// body belongs to a WHILE node) set its condition.  FCG: the iteration's delta becomes the next
// iteration's previous delta (the body always uses the slots of an even iteration k >= 2).
__global__ void loop_cond_kernel(cudaGraphConditionalHandle h, int set_handle, double* s, LoopRule r, int s_rn,
                                 int s_delta, int s_delta_prev) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  s[S_LCOUNT] += 1.0;
  if (r.kind == LOOP_FAS) {
    s[S_LREL] = s[S_RNORM] / s[S_FNORM];
  } else if (r.kind == LOOP_PF) {
    s[S_LREL] = s[S_RNORM] / s[S_FDNORM];
  } else {
    const double fn = s[S_FNORM];
    s[S_LREL] = fn != 0.0 ? s[s_rn] / fn : 1.0;
    s[s_delta_prev] = s[s_delta];
  }
  if (set_handle) cudaGraphSetConditional(h, loop_go(r, s));
}

// Flexible PCG from t >= 1: the recursive residual is trusted until it passes the test; then the true
// residual f - K x is computed and confirms or replaces it (the same rule as the host-driven loop).
__global__ void fcg_check_kernel(cudaGraphConditionalHandle h, const double* s, double tol, int s_rn) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double fn = s[S_FNORM];
  cudaGraphSetConditional(h, (fn != 0.0 && s[s_rn] / fn <= tol) ? 1u : 0u);
}
__global__ void count_true_kernel(double* s) {
  if (threadIdx.x == 0 && blockIdx.x == 0) s[S_LTRUE] += 1.0;
}

__global__ void set_scalar_kernel(double* s, int slot, double v) {
  if (threadIdx.x == 0 && blockIdx.x == 0) s[slot] = v;
}

// ---------------------------------------------------------------- graph building helpers
// Captures fn's launches on the context's stream into graph g (after deps); returns the node the
// capture ended on (null if it captured nothing) and the kernels it launched.
template <class Fn>
int capture_into(hpc_ctx* c, cudaGraph_t g, const cudaGraphNode_t* deps, size_t ndeps, Fn fn, cudaGraphNode_t* last,
                 long long* kernels) {
  const long long k0 = c->launches;
  HPC_CUDA(cudaStreamBeginCaptureToGraph(c->stream, g, deps, nullptr, ndeps, cudaStreamCaptureModeThreadLocal));
  int rc = fn();
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  const cudaGraphNode_t* cur = nullptr;
  size_t ncur = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(c->stream, &st, nullptr, nullptr, &cur, &ncur);
  if (last) *last = (e == cudaSuccess && ncur == 1) ? cur[0] : nullptr;
  const bool joined = ncur <= 1;
  cudaGraph_t out = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(c->stream, &out);
  if (kernels) *kernels = c->launches - k0;
  c->launches = k0;  // counted when the graph runs
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamGetCaptureInfo");
  if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
  if (!joined) {
    set_error("batched solve: a captured segment ended on more than one node");
    return HPC_ERR_CUDA;
  }
  return HPC_OK;
}

// A conditional node (IF or WHILE) on `handle` after `dep` in g; returns the node and its body graph.
// The handle is created first (cond_handle), so that the kernel setting it can be captured before the
// node; its value is reset to 0 at every launch of the graph.
int cond_handle(cudaGraph_t g, cudaGraphConditionalHandle* h) {
  HPC_CUDA(cudaGraphConditionalHandleCreate(h, g, 0, cudaGraphCondAssignDefault));
  return HPC_OK;
}
int add_conditional(cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalNodeType type, cudaGraphConditionalHandle h,
                    cudaGraphNode_t* node, cudaGraph_t* body) {
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = type;
  p.conditional.size = 1;
  HPC_CUDA(cudaGraphAddNode(node, g, dep ? &dep : nullptr, dep ? 1 : 0, &p));
  *body = p.conditional.phGraph_out[0];
  return HPC_OK;
}

// Launch accounting of one specimen's chain: kernels outside the loops, per body run, per
// true-residual recomputation.
struct ChainCount {
  long long fixed = 0, first = 0, body = 0, truer = 0;
};

// Common set-up of a solve on one specimen, enqueued on its stream: everything before the loop.
// Keeps the context's kernel choices as hpc_step has them during the loop (precomputed Gauss-point
// moduli active; no event timing, no nested graph replays inside the captured bodies).
struct CaptureScope {
  hpc_ctx* c;
  int graphs, timing;
  explicit CaptureScope(hpc_ctx* ctx) : c(ctx), graphs(ctx->use_graphs), timing(ctx->timing_class) {
    c->use_graphs = 0;
    c->timing_class = HPC_KC_NONE;
  }
  ~CaptureScope() {
    c->use_graphs = graphs;
    c->timing_class = timing;
  }
};

// ---------------------------------------------------------------- per-specimen solve pieces
// The mechanical solve before its loop (u_entire_dev / u_entire_fcg_dev up to the first test).
int mech_pre(hpc_ctx* c, const hpc_step_params& p) {
  int rc;
  const int L = c->maxlevel;
  const double small_k = p.small_k, Ut = 1.0;
  const bool fcg = p.mech_solver != HPC_MECH_FAS;
  if (fcg) {
    if ((rc = ensure_fcg(c))) return rc;
    if (p.mg_u.ncy + 1 > kMaxRelax) {
      set_error("ncy too large");
      return HPC_ERR_ARG;
    }
  }
  if ((rc = launch_set_scalar(c, S_FNORM, c->f_norm))) return rc;
  if ((rc = mech_material(c, small_k))) return rc;
  if ((rc = mech_diags_enqueue(c, L, small_k))) return rc;  // zero check after every specimen's set-up
  if (L > 0 && (rc = gp_material(c, small_k))) return rc;
  if (!fcg) {  // Initial_residual_u (mechanical_pcg.cpp:193-220)
    MechCall m{};
    m.level = L;
    m.finest = true;
    m.epi = EPI_RESIDUAL;
    m.src = c->F[L].u;
    m.out = c->F[L].ru;
    m.small_k = small_k;
    m.fu = c->F[L].fu;
    m.s_out0 = m.s_out1 = -1;
    m.s_out2 = S_RNORM;
    return launch_mech(c, m);
  }
  if (p.mech_solver == HPC_MECH_MIXED) {
    if ((rc = ensure_f32(c))) return rc;
    if ((rc = f32_material(c))) return rc;
  }
  LevelFields& F = c->F[L];
  const size_t vbytes = sizeof(double) * 3 * (size_t)c->L[L].n;
  if ((rc = launch_bc(c, L, F.u, nullptr, 0, Ut))) return rc;
  HPC_CUDA(cudaMemcpyAsync(c->fcg.x, F.u, vbytes, cudaMemcpyDeviceToDevice, c->stream));
  HPC_CUDA(cudaMemcpyAsync(c->fcg.f, F.fu, vbytes, cudaMemcpyDeviceToDevice, c->stream));
  return fcg_residual(c, small_k, p.t, slot_frn(-1));
}

// Loop scalars of a context after its solve graph: slots 0 .. S_LTRUE in one read.
constexpr int kLoopRead = S_LTRUE + 1;

// The mechanical solve after its loop: f_norm, the reactions (u_entire_dev / u_entire_fcg_dev).
int mech_post(hpc_ctx* c, const hpc_step_params& p, const double* sc, int* cycles, long long* fin_iters) {
  const int L = c->maxlevel;
  *cycles = (int)sc[S_LCOUNT];
  *fin_iters = (long long)*cycles * (L == 0 ? p.mg_u.nu0 : p.mg_u.nu1 + p.mg_u.nu2);
  c->f_norm = sc[S_FNORM];
  LevelFields& F = c->F[L];
  if (p.mech_solver == HPC_MECH_FAS && sc[S_ERR] != 0.0) {
    launch_set_scalar(c, S_ERR, 0.0);
    set_error("a bounded wait in a kernel (tensor copy) ran out");
    return HPC_ERR_CUDA;
  }
  if (p.mech_solver != HPC_MECH_FAS) {
    if (sc[S_ERR] != 0.0) {
      launch_set_scalar(c, S_ERR, 0.0);
      set_error("a bounded wait in a kernel (tensor copy or MMA completion) ran out");
      return HPC_ERR_CUDA;
    }
    const size_t vbytes = sizeof(double) * 3 * (size_t)c->L[L].n;
    HPC_CUDA(cudaMemcpyAsync(F.u, c->fcg.x, vbytes, cudaMemcpyDeviceToDevice, c->stream));
    HPC_CUDA(cudaMemcpyAsync(F.fu, c->fcg.f, vbytes, cudaMemcpyDeviceToDevice, c->stream));
  }
  // externe_force_nodal (mechanical_right_hnd.cpp:18-38)
  int rc;
  if ((rc = launch_bc(c, L, F.u, nullptr, 0, 1.0))) return rc;
  MechCall r{};
  r.level = L;
  r.finest = true;
  r.epi = EPI_REACTION;
  r.src = F.u;
  r.out = F.fu;
  r.small_k = p.small_k;
  r.s_out0 = r.s_out1 = r.s_out2 = -1;
  return launch_mech(c, r);
}

// The phase-field solve before its loop (phase_field_dev up to the first test).
int pf_pre(hpc_ctx* c, const hpc_step_params& p) {
  int rc;
  const int L = c->maxlevel;
  if ((rc = launch_set_scalar(c, S_FDNORM, c->fd_norm))) return rc;
  if ((rc = pf_diags_enqueue(c, L, p.lc))) return rc;  // zero check after every specimen's set-up
  PfCall m{};  // initial_residual (phase_field_pcg.cpp:106-131)
  m.level = L;
  m.epi = EPI_RESIDUAL;
  m.src = c->F[L].d;
  m.out = c->F[L].R;
  m.lc = p.lc;
  m.fd = c->F[L].fd;
  m.s_out0 = -1;
  m.s_out1 = S_RNORM;
  m.s_out2 = -1;
  return launch_pf(c, m);
}

void pf_post(hpc_ctx* c, const hpc_step_params& p, const double* sc, int* cycles, long long* fin_iters) {
  const int L = c->maxlevel;
  *cycles = (int)sc[S_LCOUNT];
  *fin_iters = (long long)*cycles * (L == 0 ? p.mg_d.nu0 : p.mg_d.nu1 + p.mg_d.nu2 * p.mg_d.nu2);
  c->fd_norm = sc[S_FDNORM];
}

// ---------------------------------------------------------------- one specimen's loop chain
// Builds, in graph g, the chain of one specimen's solve: gate -> WHILE{body; cond} (FAS, PF) or
// gate -> IF{first iteration; test; cond} -> rearm -> WHILE{iteration; test; cond} (FCG).
int build_chain(hpc_ctx* c, cudaGraph_t g, int phase, const hpc_step_params& p, ChainCount* cnt) {
  int rc;
  CaptureScope scope(c);
  const int L = c->maxlevel;
  const bool pf = phase == 1;
  const bool fcg = !pf && p.mech_solver != HPC_MECH_FAS;
  const bool mixed = p.mech_solver == HPC_MECH_MIXED;
  LoopRule rule{pf ? LOOP_PF : (fcg ? LOOP_FCG : LOOP_FAS), pf ? p.mg_d.ncy : p.mg_u.ncy, p.t,
                pf ? p.pf_tol : p.mech_tol};
  const hpc_mg& mg = pf ? p.mg_d : p.mg_u;
  const double small_k = p.small_k;
  const int kb = 2;  // the slots of an even iteration k >= 2 for every loop body
  const int k_slots[2] = {0, kb};

  cudaGraphConditionalHandle hloop = 0;
  cudaGraphNode_t gate = nullptr, loop = nullptr, prev = nullptr;
  cudaGraph_t body = nullptr;
  long long k = 0;

  // the test that ends a flexible-PCG iteration k (its residual norm in slot_frn(k))
  auto fcg_test = [&](cudaGraph_t bg, cudaGraphNode_t after, int kk, cudaGraphNode_t* out_last, long long* kern,
                      long long* truek) -> int {
    int r2;
    if (p.t == 0) {  // the true residual every iteration (f_norm follows the current reactions)
      return capture_into(c, bg, &after, 1, [&]() -> int { return fcg_residual(c, small_k, 0, slot_frn(kk)); }, out_last, kern);
    }
    cudaGraphConditionalHandle hc = 0;
    cudaGraphNode_t check = nullptr, ifn = nullptr;
    cudaGraph_t ib = nullptr;
    if ((r2 = cond_handle(bg, &hc))) return r2;
    long long kc = 0;
    if ((r2 = capture_into(c, bg, &after, 1, [&]() -> int {
           fcg_check_kernel<<<1, 32, 0, c->stream>>>(hc, c->scal, p.mech_tol, slot_frn(kk));
           HPC_CHECK_LAUNCH(c);
           return HPC_OK;
         }, &check, &kc)))
      return r2;
    if ((r2 = add_conditional(bg, check, cudaGraphCondTypeIf, hc, &ifn, &ib))) return r2;
    long long kt = 0;
    if ((r2 = capture_into(c, ib, nullptr, 0, [&]() -> int {
           int r3 = fcg_residual(c, small_k, p.t, slot_frn(kk));
           if (r3) return r3;
           count_true_kernel<<<1, 32, 0, c->stream>>>(c->scal);
           HPC_CHECK_LAUNCH(c);
           return HPC_OK;
         }, nullptr, &kt)))
      return r2;
    *kern += kc;
    *truek = kt;
    *out_last = ifn;
    return HPC_OK;
  };

  // gate: initial state, and the condition of the first loop node
  const bool first_if = fcg;  // the flexible PCG's first iteration differs (beta = 0, no gamma)
  if ((rc = cond_handle(g, &hloop))) return rc;
  if ((rc = capture_into(c, g, nullptr, 0, [&]() -> int {
         loop_gate_kernel<<<1, 32, 0, c->stream>>>(hloop, c->scal, rule, slot_frn(-1));
         HPC_CHECK_LAUNCH(c);
         return HPC_OK;
       }, &gate, &k)))
    return rc;
  cnt->fixed += k;
  if ((rc = add_conditional(g, gate, first_if ? cudaGraphCondTypeIf : cudaGraphCondTypeWhile, hloop, &loop, &body)))
    return rc;

  if (!fcg) {  // V-cycle, residual norm, condition
    const int Lr = L;
    long long kb_ = 0, kc = 0;
    cudaGraphNode_t last = nullptr;
    if ((rc = capture_into(c, body, nullptr, 0, [&]() -> int {
           int r2;
           if (pf) {
             if ((r2 = cycle_d_top(c, mg, p.lc, false))) return r2;
             return launch_dot(c, Lr, 1, c->F[Lr].R, nullptr, S_RNORM);
           }
           if ((r2 = cycle_u_top(c, mg, small_k, 1.0, p.t, false))) return r2;
           return launch_dot(c, Lr, 3, c->F[Lr].ru, nullptr, S_RNORM);
         }, &last, &kb_)))
      return rc;
    if ((rc = capture_into(c, body, &last, 1, [&]() -> int {
           loop_cond_kernel<<<1, 32, 0, c->stream>>>(hloop, 1, c->scal, rule, 0, 0, 0);
           HPC_CHECK_LAUNCH(c);
           return HPC_OK;
         }, nullptr, &kc)))
      return rc;
    cnt->body = kb_ + kc;
    return HPC_OK;
  }

  // flexible PCG: IF{iteration 0; test; cond} -> rearm -> WHILE{iteration (even slots); test; cond}
  for (int pass = 0; pass < 2; ++pass) {
    const int kk = k_slots[pass];
    cudaGraph_t bg = body;
    cudaGraphConditionalHandle hb = hloop;
    if (pass == 1) {
      cudaGraphNode_t rearm = nullptr, wn = nullptr;
      cudaGraphConditionalHandle hw = 0;
      if ((rc = cond_handle(g, &hw))) return rc;
      if ((rc = capture_into(c, g, &prev, 1, [&]() -> int {
             loop_rearm_kernel<<<1, 32, 0, c->stream>>>(hw, c->scal, rule);
             HPC_CHECK_LAUNCH(c);
             return HPC_OK;
           }, &rearm, &k)))
        return rc;
      cnt->fixed += k;
      if ((rc = add_conditional(g, rearm, cudaGraphCondTypeWhile, hw, &wn, &bg))) return rc;
      hb = hw;
    }
    long long ki = 0, kt = 0, kc = 0, ktrue = 0;
    cudaGraphNode_t it_last = nullptr, test_last = nullptr;
    if ((rc = capture_into(c, bg, nullptr, 0, [&]() -> int { return fcg_iteration(c, mg, small_k, kk, mixed, false); },
                           &it_last, &ki)))
      return rc;
    if ((rc = fcg_test(bg, it_last, kk, &test_last, &kt, &ktrue))) return rc;
    if ((rc = capture_into(c, bg, &test_last, 1, [&]() -> int {
           loop_cond_kernel<<<1, 32, 0, c->stream>>>(hb, pass == 1 ? 1 : 0, c->scal, rule, slot_frn(kk),
                                                     slot_fdelta(kk), slot_fdelta(kk + 1));
           HPC_CHECK_LAUNCH(c);
           return HPC_OK;
         }, nullptr, &kc)))
      return rc;
    if (pass == 0) {
      cnt->first = ki + kt + kc;
      prev = loop;
    } else {
      cnt->body = ki + kt + kc;
    }
    cnt->truer = ktrue;
  }
  return HPC_OK;
}

}  // namespace

int launch_set_scalar(hpc_ctx* c, int slot, double v) {
  set_scalar_kernel<<<1, 32, 0, c->stream>>>(c->scal, slot, v);
  HPC_CHECK_LAUNCH(c);
  return HPC_OK;
}

}  // namespace hpc

using namespace hpc;

// One graph per phase (mechanical, phase field) of a batch composition, rebuilt when the composition
// or any specimen's loop parameters change.
struct hpc_batch {
  struct Phase {
    cudaGraphExec_t exec = nullptr;
    std::vector<double> key;
    std::vector<ChainCount> counts;
  } phase[2];
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<cudaEvent_t> ready;
  int device = -1;
  // host seconds spent (cumulative): set-up and outputs enqueued per specimen, graph builds, waits
  // for the graphs; graph builds and launches
  double t_host = 0.0, t_build = 0.0, t_wait = 0.0;
  long long builds = 0, launches = 0;
  int timing = 0;  // wait for each graph right after its launch (hpc_batch_timing)
};

namespace {

void phase_key(std::vector<double>& key, hpc_ctx* const* ctxs, int n, const hpc_step_params* ps, int phase) {
  key.clear();
  for (int i = 0; i < n; ++i) {
    const hpc_ctx* c = ctxs[i];
    const hpc_step_params& p = ps[i];
    const hpc_mg& mg = phase == 0 ? p.mg_u : p.mg_d;
    const double v[] = {(double)c->uid, (double)mg.nu0, (double)mg.nu1, (double)mg.nu2, (double)mg.gamma,
                        (double)mg.ncy, phase == 0 ? p.small_k : p.lc, phase == 0 ? p.mech_tol : p.pf_tol,
                        (double)(p.t == 0), (double)(phase == 0 ? p.mech_solver : 0), (double)c->tc_apply,
                        (double)c->fused_coarsest, (double)c->tma_stage, (double)c->maxlevel};
    key.insert(key.end(), v, v + sizeof(v) / sizeof(v[0]));
  }
}

int run_phase(hpc_batch* b, int phase, hpc_ctx* const* ctxs, int n, const hpc_step_params* ps) {
  hpc_batch::Phase& ph = b->phase[phase];
  std::vector<double> key;
  phase_key(key, ctxs, n, ps, phase);
  auto t0 = std::chrono::steady_clock::now();
  if (!ph.exec || key != ph.key) {
    ++b->builds;
    if (ph.exec) {
      cudaGraphExecDestroy(ph.exec);
      ph.exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    HPC_CUDA(cudaGraphCreate(&g, 0));
    ph.counts.assign(n, ChainCount{});
    for (int i = 0; i < n; ++i) {
      const int rc = build_chain(ctxs[i], g, phase, ps[i], &ph.counts[i]);
      if (rc) {
        cudaGraphDestroy(g);
        return rc;
      }
    }
    const cudaError_t e = cudaGraphInstantiate(&ph.exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      ph.exec = nullptr;
      return cuda_fail(e, "cudaGraphInstantiate(batch)");
    }
    ph.key = key;
  }
  b->t_build += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ++b->launches;
  // every specimen's set-up before the graph, the graph before every specimen's next work
  for (int i = 0; i < n; ++i) {
    HPC_CUDA(cudaEventRecord(b->ready[i], ctxs[i]->stream));
    HPC_CUDA(cudaStreamWaitEvent(b->stream, b->ready[i], 0));
  }
  HPC_CUDA(cudaGraphLaunch(ph.exec, b->stream));
  HPC_CUDA(cudaEventRecord(b->done, b->stream));
  for (int i = 0; i < n; ++i) HPC_CUDA(cudaStreamWaitEvent(ctxs[i]->stream, b->done, 0));
  if (b->timing) {  // instrumentation: the graph's own duration on the host clock
    const auto w0 = std::chrono::steady_clock::now();
    HPC_CUDA(cudaEventSynchronize(b->done));
    b->t_wait += std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
  }
  return HPC_OK;
}

// Kernels the phase's graph ran for specimen i (instrumentation), from its loop scalars.
void count_launches(hpc_batch* b, int phase, int i, hpc_ctx* c, const double* sc) {
  const ChainCount& k = b->phase[phase].counts[i];
  const long long runs = (long long)sc[S_LCOUNT];
  long long n = k.fixed + (long long)sc[S_LTRUE] * k.truer;
  if (k.first) n += runs > 0 ? k.first + (runs - 1) * k.body : 0;
  else n += runs * k.body;
  c->launches += n;
}

}  // namespace

extern "C" {

int hpc_batch_create(hpc_batch** out) {
  if (!out) {
    set_error("null output");
    return HPC_ERR_ARG;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_error("no CUDA device: the library has no CPU path");
    return HPC_ERR_NODEVICE;
  }
  hpc_batch* b = new hpc_batch();
  *out = b;
  return HPC_OK;
}

int hpc_batch_destroy(hpc_batch* b) {
  if (!b) return HPC_OK;
  if (b->device >= 0) cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto& ph : b->phase)
    if (ph.exec) cudaGraphExecDestroy(ph.exec);
  for (cudaEvent_t e : b->ready) cudaEventDestroy(e);
  if (b->done) cudaEventDestroy(b->done);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return HPC_OK;
}

static int hpc_batch_step_body(hpc_batch* b, hpc_ctx* const* ctxs, int n, const hpc_step_params* ps, double* out);

int hpc_batch_step(hpc_batch* b, hpc_ctx* const* ctxs, int n, const hpc_step_params* ps, double* out) {
  if (!b || !ctxs || !ps || !out || n < 1) {
    set_error("hpc_batch_step: bad argument");
    return HPC_ERR_ARG;
  }
  const int dev = ctxs[0]->device;
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i] || ctxs[i]->device != dev) {
      set_error("hpc_batch_step: every context must exist and live on the same device");
      return HPC_ERR_ARG;
    }
    if (ctxs[i]->slab) {  // its exchanges and collectives cannot sit inside the batch's graphs
      set_error("hpc_batch_step: a slab context steps through hpc_step");
      return HPC_ERR_ARG;
    }
    for (int j = 0; j < i; ++j)
      if (ctxs[j] == ctxs[i]) {
        set_error("hpc_batch_step: a context appears twice");
        return HPC_ERR_ARG;
      }
    const hpc_step_params& p = ps[i];
    if (p.mech_solver != HPC_MECH_FAS && p.mech_solver != HPC_MECH_FCG && p.mech_solver != HPC_MECH_MIXED) {
      set_error("hpc_batch_step: unknown mech_solver");
      return HPC_ERR_ARG;
    }
  }
  HPC_CUDA(cudaSetDevice(dev));
  if (b->device < 0) {
    b->device = dev;
    HPC_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    HPC_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
  } else if (b->device != dev) {
    set_error("hpc_batch_step: a batch serves one device");
    return HPC_ERR_ARG;
  }
  while ((int)b->ready.size() < n) {
    cudaEvent_t e;
    HPC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ready.push_back(e);
  }
  const auto h0 = std::chrono::steady_clock::now();
  const double inner0 = b->t_build + b->t_wait;
  int rc = hpc_batch_step_body(b, ctxs, n, ps, out);
  b->t_host += std::chrono::duration<double>(std::chrono::steady_clock::now() - h0).count() - (b->t_build + b->t_wait - inner0);
  return rc;
}

/* Cumulative instrumentation of a batch: out[0] host seconds outside graph builds and waits, out[1]
 * seconds building graphs, out[2] seconds waiting for graphs (measured only with waits on), out[3]
 * graph builds, out[4] graph launches.  on >= 0 turns the per-launch wait on (1) or off (0). */
int hpc_batch_timing(hpc_batch* b, int on, double* out) {
  if (!b) {
    set_error("null batch");
    return HPC_ERR_ARG;
  }
  if (on >= 0) b->timing = on != 0;
  if (out) {
    out[0] = b->t_host;
    out[1] = b->t_build;
    out[2] = b->t_wait;
    out[3] = (double)b->builds;
    out[4] = (double)b->launches;
  }
  return HPC_OK;
}

static int hpc_batch_step_body(hpc_batch* b, hpc_ctx* const* ctxs, int n, const hpc_step_params* ps, double* out) {
  int rc;
  std::vector<int> mcy(n), pcy(n);
  std::vector<long long> mit(n), pit(n);
  std::vector<double> sc((size_t)n * kLoopRead);
  // Each stage is enqueued for every specimen before any host read, so that one specimen's read does
  // not hold back the next specimen's work.
  // mechanical solves: set-up per specimen, every loop in one graph launch, reactions per specimen
  for (int i = 0; i < n; ++i)
    if ((rc = mech_pre(ctxs[i], ps[i]))) return rc;
  for (int i = 0; i < n; ++i)
    if ((rc = check_zero_diags(ctxs[i], ctxs[i]->maxlevel, "PreM_u"))) return rc;
  for (int i = 0; i < n; ++i) ctxs[i]->gpm_active = ctxs[i]->maxlevel > 0 ? 1 : 0;
  rc = run_phase(b, 0, ctxs, n, ps);
  for (int i = 0; i < n && !rc; ++i) {
    rc = read_scalars(ctxs[i], 0, kLoopRead, &sc[(size_t)i * kLoopRead]);
    if (!rc) rc = mech_post(ctxs[i], ps[i], &sc[(size_t)i * kLoopRead], &mcy[i], &mit[i]);
    if (!rc) count_launches(b, 0, i, ctxs[i], &sc[(size_t)i * kLoopRead]);
  }
  for (int i = 0; i < n; ++i) ctxs[i]->gpm_active = 0;
  if (rc) return rc;
  // history, right-hand sides, phase-field solves, maxima and outputs
  for (int i = 0; i < n; ++i) {
    if ((rc = step_mid(ctxs[i], &ps[i]))) return rc;
    if ((rc = pf_pre(ctxs[i], ps[i]))) return rc;
  }
  for (int i = 0; i < n; ++i)
    if ((rc = check_zero_diags(ctxs[i], ctxs[i]->maxlevel, "Precondition_M"))) return rc;
  if ((rc = run_phase(b, 1, ctxs, n, ps))) return rc;
  for (int i = 0; i < n; ++i) {
    if ((rc = read_scalars(ctxs[i], 0, kLoopRead, &sc[(size_t)i * kLoopRead]))) return rc;
    pf_post(ctxs[i], ps[i], &sc[(size_t)i * kLoopRead], &pcy[i], &pit[i]);
    count_launches(b, 1, i, ctxs[i], &sc[(size_t)i * kLoopRead]);
    if ((rc = step_end_enqueue(ctxs[i]))) return rc;
  }
  for (int i = 0; i < n; ++i)
    if ((rc = step_end_finish(ctxs[i], &ps[i], mcy[i], mit[i], pcy[i], pit[i], out + 8 * i))) return rc;
  return HPC_OK;
}

}  // extern "C"
