"""Serving loop on the GPU: each request's result is the same alone and in a mix (GPU).

Three fracture runs of different sizes are solved one at a time, then together with overlapping
admission (three slots, staggered arrivals); outputs of every increment and the final u, d, H must
agree bit for bit, because every context owns its stream and its deterministic kernels.
"""
import numpy as np
import pytest

from hpcrack_b200 import microstructure as ms
from hpcrack_b200 import serving as sv

pytestmark = pytest.mark.gpu


def _requests():
    shapes = [(33, 33, 33), (65, 33, 33), (33, 65, 65)]
    out = []
    for i, n in enumerate(shapes):
        w = ms.inclusion_workload(f"mix{i}", n, 300 + i, 0.2, None, 3)
        out.append(sv.Request(i, w, 3, arrival=0.05 * i))
    return out


def test_same_result_alone_and_in_mix():
    alone = {}
    for req in _requests():
        srv = sv.SolveServer(hbm_budget=8 << 30, slots=1, keep_fields=True)
        (res,) = srv.replay([req])
        alone[req.rid] = res
    srv = sv.SolveServer(hbm_budget=8 << 30, slots=3, keep_fields=True)
    mixed = srv.replay(_requests())
    assert srv.peak_active >= 2  # the runs overlapped
    for res in mixed:
        ref = alone[res.rid]
        assert res.outputs == ref.outputs, res.rid
        for k in ("u", "d", "H"):
            np.testing.assert_array_equal(res.fields[k], ref.fields[k])


def test_admission_under_tight_budget():
    reqs = _requests()
    need = max(sv.default_footprint(r.workload) for r in reqs)
    srv = sv.SolveServer(hbm_budget=need, slots=3)
    res = srv.replay(reqs)
    # never more than the budget in use; the three together do not fit, the two smaller ones may
    assert srv.peak_used <= need and srv.peak_active <= 2
    assert all(len(r.outputs) == 3 for r in res)
