"""Serving and batching of staggered fracture solves on one GPU.

A request is a whole fracture run - one specimen (image, material table, load schedule) taken
through a number of staggered increments (the loop of crack_propagation.cpp:65-121, one
``hpc_step`` per increment).  :class:`SolveServer` runs requests with continuous admission:

* admission by device footprint: a request is admitted when ``hpc_footprint`` of its hierarchy fits
  in what the HBM budget has left and a slot is free; requests are taken in arrival order (a large
  request at the head waits for memory rather than being overtaken indefinitely);
* each admitted request owns a device context (its own stream) for its whole run, so u, d and H stay
  device-resident between its increments; the worker thread of the slot drives it, and the library
  releases the interpreter lock inside every call, so the increments of different requests overlap
  on the device;
* requests arriving while others run are admitted as slots and memory free up.

Each context's kernels are deterministic and contexts share no device state, so a request's result
is the same bit for bit whether it runs alone or in a mix; ``tests/test_gpu_serving.py`` checks this.
That holds with the strip shapes of the latency model, as every context without autotuning has them.
With autotuning on (``hpc_set_autotune``) the first autotuning context to meet a level size measures
the shapes under whatever load is running then and every later autotuning context reuses them; a
different shape changes the summation order, so such a request's bits can differ between a run alone
and a run in a mix (both still meet the same stopping test).  A server that wants autotuned shapes and
bit-reproducible requests tunes every size once before admitting requests.

The solver is pluggable (``solver_factory``): the CUDA library's :class:`~hpcrack_b200.solver.Hierarchy`
in production, any object with the same ``image_material`` / ``set`` / ``voigt_all_level`` /
``step`` / ``close`` methods in host-only tests of the scheduling logic.
"""
from __future__ import annotations

import dataclasses
import threading
import time
from typing import Callable, Optional

import numpy as np

from . import microstructure as ms

H_FIELD, D_FIELD = 4, 3  # hpc_field ids of H and d


@dataclasses.dataclass
class Request:
    rid: int
    workload: ms.Workload
    increments: int
    arrival: float = 0.0        # seconds after the server's start
    footprint: int = 0          # device bytes; filled by the server when 0


@dataclasses.dataclass
class Result:
    rid: int
    outputs: list               # hpc_step out[8] per increment
    admitted: float
    finished: float
    arrival: float
    fields: Optional[dict] = None  # final finest fields when the server keeps them

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def default_factory(device: int = 0, tma: bool = True):
    from .solver import Hierarchy

    def make(w: ms.Workload):
        h = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start, device=device)
        if not tma:
            h.set_tma_staging(False)
        return h

    return make


def default_footprint(w: ms.Workload) -> int:
    from .solver import Hierarchy
    return Hierarchy.footprint(w.maxlevel, w.element_nb, x0=w.x_start)


def request_mg_u(w: ms.Workload, mech_solver: int, precision_mg: bool = True):
    """The mechanical cycle parameters of a request: the workload's for the reference's FAS cycles,
    solver.precision_mg's preconditioner cycle for the flexible forms unless precision_mg is False."""
    from .solver import precision_mg as _precision_mg
    if mech_solver != 0 and precision_mg:
        return _precision_mg(w.maxlevel, w.element_nb, w.mg_u[4])
    return w.mg_u


def prepare_request(solver, w: ms.Workload):
    """Material from the image and the pre-crack (image_input.cpp:120-282, strain_history.cpp:30-70)."""
    nx, ny, nz = w.nodes
    solver.image_material(w.image, (nx, ny, nz), w.table(), w.voxel_size)
    if w.crack:
        Hc, dc = ms.precrack_fields(w)
        solver.set(H_FIELD, w.maxlevel, Hc)
        solver.set(D_FIELD, w.maxlevel, dc)
        solver.voigt_all_level(H_FIELD)


def run_request(solver, w: ms.Workload, increments: int, mech_solver: int = 0, precision_mg: bool = True):
    """One fracture run on an allocated solver: material from the image, pre-crack, increments
    (mech_solver 0: the reference's FAS cycles, 1: flexible PCG preconditioned by one FP64 V-cycle,
    2: the precision form; the flexible forms use solver.precision_mg's cycle unless precision_mg is
    False)."""
    mg_u = request_mg_u(w, mech_solver, precision_mg)
    prepare_request(solver, w)
    outs = []
    for t in range(increments):
        outs.append(solver.step(t, mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du,
                                dU_factor=w.du_factor, mech_tol=w.mech_tol, pf_tol=w.pf_tol,
                                mech_solver=mech_solver))
    return outs


class SolveServer:
    def __init__(self, hbm_budget: int, slots: int, solver_factory: Callable = None,
                 footprint: Callable = None, keep_fields: bool = False, mech_solver: int = 0,
                 precision_mg: bool = True):
        self.budget = int(hbm_budget)
        self.slots = int(slots)
        self.factory = solver_factory or default_factory()
        self.footprint = footprint or default_footprint
        self.keep_fields = keep_fields
        self.mech_solver = int(mech_solver)
        self.precision_mg = precision_mg
        self._cv = threading.Condition()
        self._pending: list[Request] = []
        self._closed = False
        self._used = 0
        self._active = 0
        self.peak_used = 0
        self.peak_active = 0
        self.results: dict[int, Result] = {}
        self.errors: dict[int, BaseException] = {}
        self._t0 = None
        self._workers: list[threading.Thread] = []

    # ---------------------------------------------------------------- client side
    def start(self):
        self._t0 = time.perf_counter()
        for i in range(self.slots):
            th = threading.Thread(target=self._worker, name=f"slot{i}", daemon=True)
            th.start()
            self._workers.append(th)

    def now(self) -> float:
        return time.perf_counter() - self._t0

    def submit(self, req: Request):
        if req.footprint <= 0:
            req.footprint = int(self.footprint(req.workload))
        if req.footprint > self.budget:
            raise ValueError(f"request {req.rid}: footprint {req.footprint} exceeds the HBM budget {self.budget}")
        with self._cv:
            if self._closed:
                raise RuntimeError("server closed")
            self._pending.append(req)
            self._cv.notify_all()

    def close(self, timeout: float = None):
        """No more requests; waits for the admitted and pending ones to finish."""
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for th in self._workers:
            th.join(timeout)

    def replay(self, requests: list[Request]):
        """Submits `requests` at their arrival times (seconds after start) and waits for all.  Requests
        arriving at t = 0 are all queued before the server starts, so that a batch submitted at once
        is admitted at once."""
        ordered = sorted(requests, key=lambda r: r.arrival)
        at_start = [r for r in ordered if r.arrival <= 0.0]
        for req in at_start:
            req.arrival = 0.0
            self.submit(req)
        self.start()
        for req in ordered[len(at_start):]:
            delay = req.arrival - self.now()
            if delay > 0:
                time.sleep(delay)
            self.submit(req)
        self.close()
        if self.errors:
            rid, exc = next(iter(self.errors.items()))
            raise RuntimeError(f"request {rid} failed: {exc}") from exc
        return [self.results[r.rid] for r in requests]

    # ---------------------------------------------------------------- slots
    def _admit(self) -> Optional[Request]:
        with self._cv:
            while True:
                if self._pending:
                    head = self._pending[0]
                    if self._used + head.footprint <= self.budget:
                        self._pending.pop(0)
                        self._used += head.footprint
                        self._active += 1
                        self.peak_used = max(self.peak_used, self._used)
                        self.peak_active = max(self.peak_active, self._active)
                        return head
                elif self._closed:
                    return None
                self._cv.wait()

    def _release(self, req: Request):
        with self._cv:
            self._used -= req.footprint
            self._active -= 1
            self._cv.notify_all()

    def _worker(self):
        while True:
            req = self._admit()
            if req is None:
                return
            admitted = self.now()
            solver = None
            try:
                solver = self.factory(req.workload)
                outs = run_request(solver, req.workload, req.increments, self.mech_solver, self.precision_mg)
                fields = None
                if self.keep_fields:
                    L = req.workload.maxlevel
                    fields = {"u": solver.get(16, L), "d": solver.get(D_FIELD, L), "H": solver.get(H_FIELD, L)}
                self.results[req.rid] = Result(req.rid, outs, admitted, self.now(), req.arrival, fields)
            except BaseException as exc:  # reported by replay(); the slot keeps serving
                self.errors[req.rid] = exc
            finally:
                if solver is not None:
                    solver.close()
                self._release(req)


class BatchServer(SolveServer):
    """Continuous batching with the library's batched increments (hpc_batch_step).

    One engine thread owns every admitted request's context.  Each round it admits what the HBM
    budget and the slots allow (arrival order), then advances every active request by one increment
    in ONE batched call: each solve phase of all requests is one CUDA graph launch whose per-request
    loops run to their own convergence.  A request that finished its increments leaves after the
    round, and its memory and slot go to the next waiting request.  The requests' results are the same
    bits as run alone (hpc_batch_step's guarantee); latency counts from arrival to the end of the round
    that completed the request.  `batch_factory` makes the batch object (hpcrack_b200.solver.Batch by
    default; a fake in host-only tests)."""

    def __init__(self, *args, batch_factory: Callable = None, time_graphs: bool = False, **kw):
        super().__init__(*args, **kw)
        self.batch_factory = batch_factory
        self.time_graphs = time_graphs
        self.rounds = 0
        self.batch_timing = None

    def start(self):
        self._t0 = time.perf_counter()
        th = threading.Thread(target=self._engine, name="batch-engine", daemon=True)
        th.start()
        self._workers.append(th)

    def _take(self, block: bool) -> list:
        """Admits pending requests that fit (arrival order, head first); blocks for one when asked."""
        out = []
        with self._cv:
            while True:
                while self._pending and self._active < self.slots:
                    head = self._pending[0]
                    if self._used + head.footprint > self.budget:
                        break
                    self._pending.pop(0)
                    self._used += head.footprint
                    self._active += 1
                    self.peak_used = max(self.peak_used, self._used)
                    self.peak_active = max(self.peak_active, self._active)
                    out.append(head)
                if out or not block or (self._closed and not self._pending):
                    return out
                self._cv.wait()

    def _engine(self):
        from .solver import step_params
        batch = None
        active = []  # [request, solver, t, outputs, admitted]
        try:
            if self.batch_factory is None:
                from .solver import Batch
                batch = Batch()
                if self.time_graphs:
                    batch.timing(True)
            else:
                batch = self.batch_factory()
            while True:
                for req in self._take(block=not active):
                    solver = None
                    try:
                        solver = self.factory(req.workload)
                        prepare_request(solver, req.workload)
                        active.append([req, solver, 0, [], self.now()])
                    except BaseException as exc:
                        self.errors[req.rid] = exc
                        if solver is not None:
                            solver.close()
                        self._release(req)
                if not active:
                    with self._cv:
                        if self._closed and not self._pending:
                            return
                    continue
                params = []
                for req, _, t, _, _ in active:
                    w = req.workload
                    params.append(step_params(t, request_mg_u(w, self.mech_solver, self.precision_mg), w.mg_d,
                                              w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du, dU_factor=w.du_factor,
                                              mech_tol=w.mech_tol, pf_tol=w.pf_tol, mech_solver=self.mech_solver))
                outs = batch.step([a[1] for a in active], params)
                self.rounds += 1
                keep = []
                for a, o in zip(active, outs):
                    a[2] += 1
                    a[3].append(o)
                    req, solver = a[0], a[1]
                    if a[2] < req.increments:
                        keep.append(a)
                        continue
                    fields = None
                    if self.keep_fields:
                        L = req.workload.maxlevel
                        fields = {"u": solver.get(16, L), "d": solver.get(D_FIELD, L), "H": solver.get(H_FIELD, L)}
                    self.results[req.rid] = Result(req.rid, a[3], a[4], self.now(), req.arrival, fields)
                    solver.close()  # the round's graph has completed; the next round rebuilds without it
                    self._release(req)
                active = keep
        except BaseException as exc:  # reported by replay()
            for a in active:
                self.errors[a[0].rid] = exc
        finally:
            if batch is not None:
                if hasattr(batch, "timing"):
                    self.batch_timing = batch.timing()
                batch.close()
            for a in active:
                a[1].close()
                self._release(a[0])


# ------------------------------------------------------------------------------------------------
# request mixes
# ------------------------------------------------------------------------------------------------
BATCH_SIZES = (33, 65, 97, 129, 161)
SERVE_SIZES = ((65, 65, 65), (97, 97, 97), (129, 129, 129), (193, 193, 193), (257, 257, 257), (257, 129, 65))
SERVE_WEIGHTS = (0.3, 0.25, 0.2, 0.1, 0.1, 0.05)


def batch_specimen(seed: int, increments: int = 5, maxlevel: int = 3) -> ms.Workload:
    """One specimen of the batched mix: node counts per axis drawn from {33, 65, 97, 129, 161}
    independently, inclusion volume fraction in [5 %, 35 %], radii scaled to the box, materials and
    loading of the 65^3 parity configuration; element_nb = (n - 1) / 2^maxlevel per axis.  The
    hierarchy is `maxlevel` deep unless that would leave fewer than 8 elements on the shortest axis
    of the coarsest level (a 33-node axis stops at maxlevel 2): the reference's fixed 50-iteration
    coarsest PCG is not stable on smaller coarsest grids."""
    rng = np.random.default_rng(seed)
    nodes = tuple(int(rng.choice(BATCH_SIZES)) for _ in range(3))
    vf = float(rng.uniform(0.05, 0.35))
    L = min(maxlevel, ms.hierarchy_for(nodes)[0])
    return ms.inclusion_workload(f"batch{seed}", nodes, seed, vf, L, increments)


def serve_mix(n: int, rate: float, seed: int = 7, increments: int = 10, sizes=SERVE_SIZES,
              weights=SERVE_WEIGHTS) -> list[Request]:
    """Poisson arrivals at `rate` requests/s; sizes drawn with `weights`; volume fraction in
    [5 %, 35 %].  Sizes and volume fractions come from one random stream and the arrival gaps from
    another (both seeded by `seed`), so every rate serves the same requests."""
    rng = np.random.default_rng(seed)
    arr = np.random.default_rng([seed, 1])
    t = 0.0
    reqs = []
    w = np.asarray(weights, dtype=np.float64)
    w = w / w.sum()
    for i in range(n):
        t += float(arr.exponential(1.0 / rate))
        nodes = sizes[int(rng.choice(len(sizes), p=w))]
        vf = float(rng.uniform(0.05, 0.35))
        wl = ms.inclusion_workload(f"req{i}", nodes, seed * 100000 + i, vf, None, increments)
        reqs.append(Request(i, wl, increments, arrival=t))
    return reqs


def latency_stats(results: list[Result], wall: float) -> dict:
    lat = np.array([r.latency for r in results])
    return {"requests": len(results), "solves_per_s": len(results) / wall if wall > 0 else None,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "wall_s": wall}
