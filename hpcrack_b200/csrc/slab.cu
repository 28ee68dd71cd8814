// z-slab decomposition of one specimen over ranks: the per-level extents of a rank, the combination
// of its reductions over the ranks and the exchange of its ghost planes.
//
// The split follows the reference's 3-D MPI decomposition restricted to z (one rank per GPU):
//   - local node counts per level: initialize (initialization.cpp:19-134);
//   - global coordinates of local planes: get_coordinate (boundary_conditions.cpp:13-18);
//   - owned planes: realdomain (realdomain.h:17-40), reductions over them (pcg_utilities.cpp:16-58)
//     combined over the ranks (MPI_Reduce + MPI_Bcast there);
//   - ghost planes: SendRecv (mpi_communications.h:24-47): plane nz-2 to the rank above (its plane 0),
//     plane 1 to the rank below (its plane nz-1).
// Two transports carry the same operations:
//   - an in-process group: ranks are host threads of one process (one GPU or several), the planes move
//     by device copies and the reductions through host memory, between host barriers;
//   - NCCL (one process per GPU): grouped send/recv of the planes and an all-reduce of the scalars, on
//     the context's stream.  NCCL is loaded at run time, so the library has no link dependency on it.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

namespace hpc {
constexpr int kMaxSlabRanks = 64;
constexpr double kBarrierSeconds = 120.0;  // a rank that never arrives ends the others' wait with an error
}  // namespace hpc

// In-process group of slab ranks (hpc_slab_group_create).
struct hpc_slab_group {
  int nr;
  std::mutex mu;
  std::condition_variable cv;
  int arrived;
  unsigned long long gen;
  bool aborted;
  hpc_ctx* member[hpc::kMaxSlabRanks];
  // ghost exchange: each rank's array, published between the two barriers of an exchange
  struct Pub {
    const char* v;
    long long comp_bytes;  // component stride
    int nz;
  } pub[hpc::kMaxSlabRanks];
  // reductions: each rank's values, double-buffered by call parity (a rank can be at most one
  // reduction ahead of another: the next one's barrier waits for all)
  double vals[2][hpc::kMaxSlabRanks][3];
  // gathers: each rank's source arrays, published between the two barriers of a gather
  struct GatherPub {
    const char* src[8];
    long long comp_bytes;
  } gpub[hpc::kMaxSlabRanks];
};

struct NcclApi {
  bool ok;
  std::string why;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*);
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int);
  ncclResult_t (*CommDestroy)(ncclComm_t);
  ncclResult_t (*GroupStart)();
  ncclResult_t (*GroupEnd)();
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t);
  const char* (*GetErrorString)(ncclResult_t);
};

struct SlabState {
  int nr, rank;
  hpc_slab_group* group;  // in-process transport
  ncclComm_t comm;        // NCCL transport
  double* hval;           // pinned staging of the reduced scalars
  int parity;
  hpc::SlabLevel plan[hpc::kMaxSlabRanks];  // every rank's coarsest-level planes
  // the whole coarsest level, gathered for the redundant solve (allocated on first use)
  struct Coarse {
    int ready;
    hpc::LevelGeo g;
    double* base;  // u, fu, ru, invM (3 components each), Ke, Ge
    uint8_t* bz;
    double *u, *fu, *ru, *invM, *Ke, *Ge;
  } co;
};

namespace hpc {
namespace {

NcclApi& nccl() {
  static NcclApi api{};
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      api.why = std::string("NCCL not found: ") + dlerror();
      return;
    }
    bool all = true;
    auto sym = [&](auto& fn, const char* name) {
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
      all = all && fn;
    };
    sym(api.GetUniqueId, "ncclGetUniqueId");
    sym(api.CommInitRank, "ncclCommInitRank");
    sym(api.CommDestroy, "ncclCommDestroy");
    sym(api.GroupStart, "ncclGroupStart");
    sym(api.GroupEnd, "ncclGroupEnd");
    sym(api.Send, "ncclSend");
    sym(api.Recv, "ncclRecv");
    sym(api.AllReduce, "ncclAllReduce");
    sym(api.GetErrorString, "ncclGetErrorString");
    api.ok = all;
    if (!all) api.why = "NCCL library lacks a needed entry point";
  });
  return api;
}

int nccl_fail(ncclResult_t r, const char* where) {
  set_error(std::string(where) + ": " + nccl().GetErrorString(r));
  return HPC_ERR_CUDA;
}

int comm_fail(const char* what) {
  set_error(what);
  return HPC_ERR_CUDA;
}

// Host barrier of the in-process group, bounded: a rank that does not arrive within
// kBarrierSeconds (or a group aborted by a failing rank) ends every wait with an error.
int group_barrier(hpc_slab_group* g) {
  std::unique_lock<std::mutex> lock(g->mu);
  if (g->aborted) return comm_fail("slab group aborted by another rank");
  const unsigned long long my = g->gen;
  if (++g->arrived == g->nr) {
    g->arrived = 0;
    ++g->gen;
    g->cv.notify_all();
    return HPC_OK;
  }
  const bool done = g->cv.wait_for(lock, std::chrono::duration<double>(kBarrierSeconds),
                                   [&] { return g->gen != my || g->aborted; });
  if (!done || g->aborted) {
    g->aborted = true;
    g->cv.notify_all();
    return comm_fail(done ? "slab group aborted by another rank" : "slab group: a rank did not arrive in time");
  }
  return HPC_OK;
}

double combine(int op, double a, double b) {
  if (op == 1) return std::fmax(a, b);
  if (op == 2) return std::fmin(a, b);
  return a + b;
}

int local_reduce(hpc_ctx* c, const int* slots, int op) {
  SlabState* s = c->slab;
  hpc_slab_group* g = s->group;
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 3; ++k)
    if (slots[k] >= 0) HPC_CUDA(cudaMemcpy(&s->hval[k], c->scal + slots[k], sizeof(double), cudaMemcpyDeviceToHost));
  const int par = s->parity;
  s->parity ^= 1;
  for (int k = 0; k < 3; ++k) g->vals[par][s->rank][k] = slots[k] >= 0 ? s->hval[k] : 0.0;
  int rc = group_barrier(g);
  if (rc) return rc;
  for (int k = 0; k < 3; ++k) {
    if (slots[k] < 0) continue;
    double v = g->vals[par][0][k];
    for (int r = 1; r < g->nr; ++r) v = combine(op, v, g->vals[par][r][k]);  // rank order on every rank
    s->hval[k] = v;
    HPC_CUDA(cudaMemcpy(c->scal + slots[k], &s->hval[k], sizeof(double), cudaMemcpyHostToDevice));
  }
  return HPC_OK;
}

int local_halo(hpc_ctx* c, int level, char* v, int ncomp, int elem) {
  SlabState* s = c->slab;
  hpc_slab_group* g = s->group;
  const LevelGeo& L = c->L[level];
  const long long plane = L.plane * elem, comp = L.n * elem;
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  g->pub[s->rank] = hpc_slab_group::Pub{v, comp, L.nz};
  int rc = group_barrier(g);
  if (rc) return rc;
  for (int m = 0; m < ncomp; ++m) {
    if (s->rank > 0) {
      const auto& p = g->pub[s->rank - 1];
      HPC_CUDA(cudaMemcpyAsync(v + m * comp, p.v + m * p.comp_bytes + (long long)(p.nz - 2) * plane, plane,
                               cudaMemcpyDefault, c->stream));
    }
    if (s->rank < s->nr - 1) {
      const auto& p = g->pub[s->rank + 1];
      HPC_CUDA(cudaMemcpyAsync(v + m * comp + (long long)(L.nz - 1) * plane, p.v + m * p.comp_bytes + plane, plane,
                               cudaMemcpyDefault, c->stream));
    }
  }
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  return group_barrier(g);  // nobody changes its planes before every neighbour has copied them
}

int nccl_reduce(hpc_ctx* c, const int* slots, int op) {
  NcclApi& api = nccl();
  const ncclRedOp_t nop = op == 1 ? ncclMax : op == 2 ? ncclMin : ncclSum;
  ncclResult_t r = api.GroupStart();
  if (r != ncclSuccess) return nccl_fail(r, "ncclGroupStart");
  for (int k = 0; k < 3; ++k)
    if (slots[k] >= 0) {
      double* p = c->scal + slots[k];
      if ((r = api.AllReduce(p, p, 1, ncclFloat64, nop, c->slab->comm, c->stream)) != ncclSuccess) {
        api.GroupEnd();
        return nccl_fail(r, "ncclAllReduce");
      }
    }
  if ((r = api.GroupEnd()) != ncclSuccess) return nccl_fail(r, "ncclGroupEnd");
  return HPC_OK;
}

int nccl_halo(hpc_ctx* c, int level, char* v, int ncomp, int elem) {
  NcclApi& api = nccl();
  SlabState* s = c->slab;
  const LevelGeo& L = c->L[level];
  const size_t count = (size_t)L.plane;
  const long long plane = L.plane * elem, comp = L.n * elem;
  const ncclDataType_t t = elem == 8 ? ncclFloat64 : ncclFloat32;
  ncclResult_t r = api.GroupStart();
  if (r != ncclSuccess) return nccl_fail(r, "ncclGroupStart");
  for (int m = 0; m < ncomp && r == ncclSuccess; ++m) {
    char* base = v + m * comp;
    if (s->rank > 0) {
      r = api.Send(base + plane, count, t, s->rank - 1, s->comm, c->stream);
      if (r == ncclSuccess) r = api.Recv(base, count, t, s->rank - 1, s->comm, c->stream);
    }
    if (r == ncclSuccess && s->rank < s->nr - 1) {
      r = api.Send(base + (long long)(L.nz - 2) * plane, count, t, s->rank + 1, s->comm, c->stream);
      if (r == ncclSuccess) r = api.Recv(base + (long long)(L.nz - 1) * plane, count, t, s->rank + 1, s->comm, c->stream);
    }
  }
  const ncclResult_t e = api.GroupEnd();
  if (r != ncclSuccess) return nccl_fail(r, "ncclSend/ncclRecv");
  if (e != ncclSuccess) return nccl_fail(e, "ncclGroupEnd");
  return HPC_OK;
}

// Gather of the coarsest level: every rank's owned planes of `nf` fields (ncomp[f] components each)
// into the whole-level arrays dst[f] (geometry gd) of every rank.
int local_gather(hpc_ctx* c, const double* const* src, double* const* dst, const int* ncomp, int nf,
                 const LevelGeo& gd) {
  SlabState* s = c->slab;
  hpc_slab_group* g = s->group;
  const LevelGeo& L = c->L[0];
  const long long plane = L.plane * (long long)sizeof(double);
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  auto& mine = g->gpub[s->rank];
  for (int f = 0; f < nf; ++f) mine.src[f] = reinterpret_cast<const char*>(src[f]);
  mine.comp_bytes = L.n * (long long)sizeof(double);
  int rc = group_barrier(g);
  if (rc) return rc;
  for (int q = 0; q < s->nr; ++q) {
    const SlabLevel& pq = s->plan[q];
    const auto& pub = g->gpub[q];
    for (int f = 0; f < nf; ++f)
      for (int m = 0; m < ncomp[f]; ++m) {
        char* d = reinterpret_cast<char*>(dst[f]) + m * gd.n * (long long)sizeof(double) + (long long)(pq.zb + pq.lo) * plane;
        const char* from = pub.src[f] + m * pub.comp_bytes + (long long)pq.lo * plane;
        HPC_CUDA(cudaMemcpyAsync(d, from, (size_t)(pq.hi - pq.lo) * plane, cudaMemcpyDefault, c->stream));
      }
  }
  HPC_CUDA(cudaStreamSynchronize(c->stream));
  return group_barrier(g);
}

int nccl_gather(hpc_ctx* c, const double* const* src, double* const* dst, const int* ncomp, int nf,
                const LevelGeo& gd) {
  NcclApi& api = nccl();
  SlabState* s = c->slab;
  const LevelGeo& L = c->L[0];
  const SlabLevel& me = s->plan[s->rank];
  for (int f = 0; f < nf; ++f)  // this rank's own planes
    for (int m = 0; m < ncomp[f]; ++m)
      HPC_CUDA(cudaMemcpyAsync(dst[f] + m * gd.n + (me.zb + me.lo) * L.plane, src[f] + m * L.n + me.lo * L.plane,
                               sizeof(double) * (size_t)(me.hi - me.lo) * L.plane, cudaMemcpyDeviceToDevice, c->stream));
  ncclResult_t r = api.GroupStart();
  if (r != ncclSuccess) return nccl_fail(r, "ncclGroupStart");
  for (int f = 0; f < nf && r == ncclSuccess; ++f)
    for (int m = 0; m < ncomp[f] && r == ncclSuccess; ++m)
      for (int q = 0; q < s->nr && r == ncclSuccess; ++q) {
        if (q == s->rank) continue;
        const SlabLevel& pq = s->plan[q];
        r = api.Send(src[f] + m * L.n + me.lo * L.plane, (size_t)(me.hi - me.lo) * L.plane, ncclFloat64, q, s->comm,
                     c->stream);
        if (r == ncclSuccess)
          r = api.Recv(dst[f] + m * gd.n + (pq.zb + pq.lo) * L.plane, (size_t)(pq.hi - pq.lo) * L.plane, ncclFloat64,
                       q, s->comm, c->stream);
      }
  const ncclResult_t e = api.GroupEnd();
  if (r != ncclSuccess) return nccl_fail(r, "ncclSend/ncclRecv (gather)");
  if (e != ncclSuccess) return nccl_fail(e, "ncclGroupEnd");
  return HPC_OK;
}

int no_transport() {
  set_error("slab context of several ranks without a transport (hpc_slab_group_join or hpc_slab_join_nccl)");
  return HPC_ERR_ARG;
}

}  // namespace

bool slab_levels(const hpc_geometry& g, int nr, int r, SlabLevel* out) {
  if (nr < 1 || nr > kMaxSlabRanks || r < 0 || r >= nr || g.maxlevel < 0 || g.maxlevel >= kMaxLevels) return false;
  const int K0 = g.element_nb[2] + 1;  // coarsest nodes along z
  const int q = K0 / nr, rem = K0 % nr;
  if (q < 1) return false;
  const bool first = nr == 1 || r == 0, last = nr == 1 || r == nr - 1;
  int n = nr == 1 ? K0 : r == 0 ? q + 1 : r == nr - 1 ? q + rem + 1 : q + 2;
  long long kk = g.element_nb[2];  // elements along z on the level
  for (int l = 0; l <= g.maxlevel; ++l) {
    SlabLevel& s = out[l];
    s.nz = n;
    s.zb = first ? 0 : (r == nr - 1) ? (int)(kk - n + 1) : r * (n - 2) - 1;
    s.lo = first ? 0 : 1;
    s.hi = last ? n : n - 1;
    kk *= 2;
    n = first ? 2 * (n - 1) + 1 : (r == nr - 1) ? 2 * (n - 1) : 2 * (n - 2) + 2;
  }
  return true;
}

int slab_after_launch(hpc_ctx* c) {
  if (!c->red_pending) return HPC_OK;
  c->red_pending = 0;
  const int* slots = c->red_slot;
  if (slots[0] < 0 && slots[1] < 0 && slots[2] < 0) return HPC_OK;
  SlabState* s = c->slab;
  if (s->nr == 1 && !s->comm) return HPC_OK;
  if (s->group) return local_reduce(c, slots, c->red_op);
  if (s->comm) return nccl_reduce(c, slots, c->red_op);
  return no_transport();
}

int slab_halo(hpc_ctx* c, int level, void* v, int ncomp, int elem_bytes) {
  SlabState* s = c->slab;
  if (s->nr == 1) return HPC_OK;
  if (s->group) return local_halo(c, level, static_cast<char*>(v), ncomp, elem_bytes);
  if (s->comm) return nccl_halo(c, level, static_cast<char*>(v), ncomp, elem_bytes);
  return no_transport();
}

int slab_coarsest_mode(hpc_ctx* c) {
  if (!c->slab || c->slab->nr == 1) return 0;
  LevelGeo g = c->L[0];
  g.nz = c->geo.element_nb[2] + 1;
  return c->maxlevel > 0 && coarse_pcg_fits_geo(g) ? 1 : 2;
}

int slab_coarsest(hpc_ctx* c, double Ut, int nb) {
  SlabState* s = c->slab;
  auto& co = s->co;
  const LevelGeo& L = c->L[0];
  if (!co.ready) {
    LevelGeo g = L;
    g.nz = c->geo.element_nb[2] + 1;
    g.n = g.plane * g.nz;
    g.zb = 0;
    g.oz0 = 0;
    g.oz1 = g.nz;
    g.zsh = 0;
    std::vector<uint8_t> fz(g.nz);
    const double* B = c->box;
    for (int k = 0; k < g.nz; ++k) {  // the Dirichlet planes of the whole level, as hpc_create sets them
      const double z = B[4] + k * g.hz;
      fz[k] = (uint8_t)((z == B[4] ? 1 : 0) | (z == B[5] ? 2 : 0));
    }
    const size_t doubles = (size_t)g.n * 14;
    HPC_CUDA(cudaMallocAsync((void**)&co.base, sizeof(double) * doubles + g.nz, c->stream));
    HPC_CUDA(cudaMemsetAsync(co.base, 0, sizeof(double) * doubles, c->stream));
    co.u = co.base;
    co.fu = co.u + 3 * g.n;
    co.ru = co.fu + 3 * g.n;
    co.invM = co.ru + 3 * g.n;
    co.Ke = co.invM + 3 * g.n;
    co.Ge = co.Ke + g.n;
    co.bz = reinterpret_cast<uint8_t*>(co.base + doubles);
    HPC_CUDA(cudaMemcpyAsync(co.bz, fz.data(), g.nz, cudaMemcpyHostToDevice, c->stream));
    HPC_CUDA(cudaStreamSynchronize(c->stream));  // fz leaves scope
    g.bz = co.bz;
    co.g = g;
    co.ready = 1;
  }
  const LevelFields& F = c->F[0];
  const double* src[5] = {F.u, F.fu, F.preMu, F.Ke, F.Ge};
  double* dst[5] = {co.u, co.fu, co.invM, co.Ke, co.Ge};
  const int nc[5] = {3, 3, 3, 1, 1};
  int rc = s->group ? local_gather(c, src, dst, nc, 5, co.g) : s->comm ? nccl_gather(c, src, dst, nc, 5, co.g) : no_transport();
  if (rc) return rc;
  // the same inputs on every rank, a deterministic solver: the same whole-level solution everywhere
  if ((rc = launch_coarse_pcg_on(c, co.g, co.u, co.fu, co.ru, co.invM, co.Ke, co.Ge, Ut, nb))) return rc;
  for (int m = 0; m < 3; ++m) {  // this rank's planes, ghost planes included
    HPC_CUDA(cudaMemcpyAsync(F.u + m * L.n, co.u + m * co.g.n + L.zb * L.plane, sizeof(double) * L.n,
                             cudaMemcpyDeviceToDevice, c->stream));
    HPC_CUDA(cudaMemcpyAsync(F.ru + m * L.n, co.ru + m * co.g.n + L.zb * L.plane, sizeof(double) * L.n,
                             cudaMemcpyDeviceToDevice, c->stream));
  }
  return HPC_OK;
}

void slab_release(hpc_ctx* c) {
  SlabState* s = c->slab;
  if (!s) return;
  if (s->co.base) cudaFreeAsync(s->co.base, c->stream);
  if (s->group) {
    std::lock_guard<std::mutex> lock(s->group->mu);
    if (s->group->member[s->rank] == c) s->group->member[s->rank] = nullptr;
  }
  if (s->comm) nccl().CommDestroy(s->comm);
  if (s->hval) cudaFreeHost(s->hval);
  delete s;
  c->slab = nullptr;
}

// Attaches the slab state to a context just created for rank r of nr (hpcrack.cu).
int slab_attach(hpc_ctx* c, int nr, int r) {
  SlabState* s = new SlabState();
  s->nr = nr;
  s->rank = r;
  c->slab = s;
  for (int q = 0; q < nr; ++q) {
    SlabLevel lv[kMaxLevels];
    if (!slab_levels(c->geo, nr, q, lv)) {
      set_error("bad slab decomposition");
      return HPC_ERR_ARG;
    }
    s->plan[q] = lv[0];
  }
  HPC_CUDA(cudaMallocHost((void**)&s->hval, sizeof(double) * 4));
  return HPC_OK;
}

}  // namespace hpc

using namespace hpc;

extern "C" {

int hpc_slab_level(const hpc_geometry* geo, int nranks, int rank, int level, int* out4) {
  SlabLevel lv[kMaxLevels];
  if (!geo || !out4 || !slab_levels(*geo, nranks, rank, lv) || level < 0 || level > geo->maxlevel) {
    set_error("bad slab decomposition (every rank needs at least one coarsest plane)");
    return HPC_ERR_ARG;
  }
  out4[0] = lv[level].nz;
  out4[1] = lv[level].zb;
  out4[2] = lv[level].lo;
  out4[3] = lv[level].hi;
  return HPC_OK;
}

int hpc_slab_group_create(hpc_slab_group** out, int nranks) {
  if (!out || nranks < 1 || nranks > kMaxSlabRanks) {
    set_error("bad slab group size");
    return HPC_ERR_ARG;
  }
  hpc_slab_group* g = new hpc_slab_group();
  g->nr = nranks;
  g->arrived = 0;
  g->gen = 0;
  g->aborted = false;
  for (int r = 0; r < kMaxSlabRanks; ++r) g->member[r] = nullptr;
  *out = g;
  return HPC_OK;
}

int hpc_slab_group_join(hpc_slab_group* g, hpc_ctx* c) {
  if (!g || !c || !c->slab || c->slab->nr != g->nr || c->slab->group || c->slab->comm) {
    set_error("slab group join: context is not a free slab rank of this group's size");
    return HPC_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g->mu);
  if (g->member[c->slab->rank]) {
    set_error("slab group join: rank already taken");
    return HPC_ERR_ARG;
  }
  g->member[c->slab->rank] = c;
  c->slab->group = g;
  return HPC_OK;
}

int hpc_slab_group_abort(hpc_slab_group* g) {
  if (!g) return HPC_ERR_ARG;
  std::lock_guard<std::mutex> lock(g->mu);
  g->aborted = true;
  g->cv.notify_all();
  return HPC_OK;
}

int hpc_slab_group_destroy(hpc_slab_group* g) {
  if (!g) return HPC_OK;
  {
    std::lock_guard<std::mutex> lock(g->mu);
    for (int r = 0; r < g->nr; ++r)
      if (g->member[r]) {
        set_error("slab group destroyed while a member context lives");
        return HPC_ERR_ARG;
      }
  }
  delete g;
  return HPC_OK;
}

int hpc_nccl_unique_id(unsigned char* out128) {
  if (!out128) return HPC_ERR_ARG;
  NcclApi& api = nccl();
  if (!api.ok) {
    set_error(api.why);
    return HPC_ERR_NODEVICE;
  }
  ncclUniqueId id;
  const ncclResult_t r = api.GetUniqueId(&id);
  if (r != ncclSuccess) return nccl_fail(r, "ncclGetUniqueId");
  static_assert(sizeof(id.internal) == 128, "NCCL unique id size");
  std::memcpy(out128, id.internal, 128);
  return HPC_OK;
}

int hpc_slab_join_nccl(hpc_ctx* c, const unsigned char* id128) {
  if (!c || !c->slab || !id128 || c->slab->group || c->slab->comm) {
    set_error("NCCL join: context is not a free slab rank");
    return HPC_ERR_ARG;
  }
  NcclApi& api = nccl();
  if (!api.ok) {
    set_error(api.why);
    return HPC_ERR_NODEVICE;
  }
  cudaSetDevice(c->device);
  ncclUniqueId id;
  std::memcpy(id.internal, id128, 128);
  ncclComm_t comm = nullptr;
  const ncclResult_t r = api.CommInitRank(&comm, c->slab->nr, id, c->slab->rank);
  if (r != ncclSuccess) return nccl_fail(r, "ncclCommInitRank");
  c->slab->comm = comm;
  // NCCL's calls are enqueued on the stream without host waits, so the coarse parts of the cycles
  // may be captured into graphs with them inside (the first cycle, uncaptured, sets up the peers)
  c->use_graphs = 1;
  return HPC_OK;
}

}  // extern "C"
