"""Host logic of the serving loop: admission by footprint, arrival order, slot reuse, error
reporting, request mixes (no GPU: a fake solver stands in for the device context)."""
import threading
import time

import numpy as np
import pytest

from hpcrack_b200 import microstructure as ms
from hpcrack_b200 import serving as sv


class FakeSolver:
    """Same methods as Hierarchy; each increment sleeps and returns values derived from the
    workload so results identify their request."""
    live = 0
    lock = threading.Lock()

    def __init__(self, w, fail=False):
        self.w = w
        self.fail = fail
        with FakeSolver.lock:
            FakeSolver.live += 1

    def image_material(self, *a):
        pass

    def set(self, *a):
        pass

    def voigt_all_level(self, *a):
        pass

    def step(self, t, *a, **k):
        if self.fail:
            raise RuntimeError("solver failure")
        time.sleep(0.01)
        return [float(t), float(self.w.image.sum()), 0, 0, 1, 1, 6, 3]

    def close(self):
        with FakeSolver.lock:
            FakeSolver.live -= 1


def _req(rid, n, arrival=0.0, increments=2, footprint=10):
    w = ms.inclusion_workload(f"r{rid}", (n, n, n), rid, 0.1, 0, increments)
    return sv.Request(rid, w, increments, arrival=arrival, footprint=footprint)


def test_admission_respects_budget_and_slots():
    reqs = [_req(i, 9, arrival=0.0, footprint=[40, 30, 50, 20, 60][i]) for i in range(5)]
    srv = sv.SolveServer(hbm_budget=100, slots=3, solver_factory=FakeSolver)
    res = srv.replay(reqs)
    assert [r.rid for r in res] == [0, 1, 2, 3, 4]
    assert srv.peak_used <= 100 and srv.peak_active <= 3
    assert FakeSolver.live == 0
    for r in res:
        assert len(r.outputs) == 2 and r.finished >= r.admitted >= 0.0
        assert r.outputs[0][1] == float(reqs[r.rid].workload.image.sum())
    # arrival order: request 2 (50) cannot start before 0 and 1 leave room, request 4 comes last
    order = sorted(res, key=lambda r: r.admitted)
    assert order[0].rid in (0, 1) and order[-1].rid == 4


def test_oversized_request_is_refused():
    srv = sv.SolveServer(hbm_budget=100, slots=1, solver_factory=FakeSolver)
    srv.start()
    with pytest.raises(ValueError, match="exceeds the HBM budget"):
        srv.submit(_req(0, 9, footprint=101))
    srv.close()


def test_failed_request_is_reported_and_slot_survives():
    def factory(w):
        return FakeSolver(w, fail=(w.name == "r1"))

    srv = sv.SolveServer(hbm_budget=100, slots=1, solver_factory=factory)
    with pytest.raises(RuntimeError, match="request 1 failed"):
        srv.replay([_req(0, 9), _req(1, 9), _req(2, 9)])
    assert set(srv.results) == {0, 2}
    assert FakeSolver.live == 0


def test_latency_stats_and_mixes():
    reqs = sv.serve_mix(50, rate=20.0, seed=7, increments=10)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0) and 1.0 < arr[-1] < 5.0  # ~50 / 20 s
    sizes = [r.workload.nodes for r in reqs]
    assert set(sizes) <= set(sv.SERVE_SIZES)
    again = sv.serve_mix(50, rate=20.0, seed=7, increments=10)
    assert [r.workload.nodes for r in again] == sizes
    other_rate = sv.serve_mix(50, rate=5.0, seed=7, increments=10)  # the same requests at every rate
    assert [r.workload.nodes for r in other_rate] == sizes
    assert np.array_equal(other_rate[3].workload.image, reqs[3].workload.image)
    b = sv.batch_specimen(100)
    assert all(n in sv.BATCH_SIZES for n in b.nodes)
    assert all(e << b.maxlevel == n - 1 for e, n in zip(b.element_nb, b.nodes))
    assert min(b.element_nb) >= 8
    res = [sv.Result(i, [], 0.0, 1.0 + i, 0.0) for i in range(100)]
    st = sv.latency_stats(res, wall=10.0)
    assert st["solves_per_s"] == 10.0 and st["p50_s"] == pytest.approx(50.5) and st["p99_s"] > 99.0


def test_hierarchy_rule():
    assert ms.hierarchy_for((257, 257, 257)) == (5, (8, 8, 8))
    assert ms.hierarchy_for((257, 129, 65)) == (3, (32, 16, 8))
    assert ms.hierarchy_for((193, 193, 193)) == (4, (12, 12, 12))


class FakeBatch:
    """Stands in for hpcrack_b200.solver.Batch: one call advances every given solver by its own t."""
    sizes = []

    def step(self, hiers, params):
        FakeBatch.sizes.append(len(hiers))
        return [h.step(p.t) for h, p in zip(hiers, params)]

    def close(self):
        pass


def test_batch_server_rounds_admission_and_results():
    """The batched engine: every round advances all active requests by one increment in one call;
    requests are admitted in arrival order within the budget and slots, leave after their last
    increment and hand their memory to the next; each result holds its own increments in order."""
    FakeBatch.sizes = []
    incs = [2, 3, 1, 2, 2]
    reqs = [_req(i, 9, arrival=0.0, footprint=[40, 30, 50, 20, 60][i], increments=incs[i]) for i in range(5)]
    srv = sv.BatchServer(hbm_budget=100, slots=3, solver_factory=FakeSolver, batch_factory=FakeBatch)
    res = srv.replay(reqs)
    assert [r.rid for r in res] == [0, 1, 2, 3, 4]
    assert srv.peak_used <= 100 and srv.peak_active <= 3
    assert FakeSolver.live == 0
    for r, n in zip(res, incs):
        assert [o[0] for o in r.outputs] == [float(t) for t in range(n)]
        assert r.outputs[0][1] == float(reqs[r.rid].workload.image.sum())
        assert r.finished >= r.admitted >= 0.0
    assert max(FakeBatch.sizes) >= 2 and srv.rounds == len(FakeBatch.sizes)
    assert sum(FakeBatch.sizes) == sum(incs)


def test_batch_server_admits_late_arrivals_between_rounds():
    FakeBatch.sizes = []
    reqs = [_req(0, 9, arrival=0.0, increments=6), _req(1, 9, arrival=0.03, increments=2)]
    srv = sv.BatchServer(hbm_budget=100, slots=4, solver_factory=FakeSolver, batch_factory=FakeBatch)
    res = srv.replay(reqs)
    assert len(res[0].outputs) == 6 and len(res[1].outputs) == 2
    assert 2 in FakeBatch.sizes  # the late request ran in the same calls as the first one
    assert res[1].admitted >= 0.03 - 1e-3


def test_batch_submitted_at_once_runs_in_one_round_per_increment():
    """Requests arriving at t = 0 are queued before the engine starts: every round holds all of them."""
    FakeBatch.sizes = []
    reqs = [_req(i, 9, arrival=0.0, increments=3) for i in range(12)]
    srv = sv.BatchServer(hbm_budget=1000, slots=12, solver_factory=FakeSolver, batch_factory=FakeBatch)
    srv.replay(reqs)
    assert FakeBatch.sizes == [12, 12, 12]


def test_batch_server_reports_a_failed_round_and_releases_every_context():
    """A batched call that fails (one context's error fails the whole hpc_batch_step) is reported for
    the requests in that round; every context is closed and its memory released."""
    class FailingBatch(FakeBatch):
        def step(self, hiers, params):
            if any(h.w.name == "r2" for h in hiers):
                raise RuntimeError("batched step failed")
            return super().step(hiers, params)

    reqs = [_req(i, 9, arrival=0.0, increments=2) for i in range(4)]
    srv = sv.BatchServer(hbm_budget=100, slots=4, solver_factory=FakeSolver, batch_factory=FailingBatch)
    with pytest.raises(RuntimeError, match="failed"):
        srv.replay(reqs)
    assert FakeSolver.live == 0
    assert srv._used == 0 and srv._active == 0
