"""Strip-shape autotuning (GPU): measured shapes change only the rounding of the reductions, so a
tuned run matches an untuned one to the parity tolerance, and the measured shapes are recorded."""
import pytest

from hpcrack_b200 import microstructure as ms
from hpcrack_b200.solver import Hierarchy
from cases import D, U, load_workload, rel

pytestmark = pytest.mark.gpu


def test_autotuned_run_matches_model_shapes():
    w = ms.make_workload("small33")
    runs = []
    for tune in (False, True):
        h = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start)
        h.set_autotune(tune)
        load_workload([h], w)
        outs = [h.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du, mech_tol=1e-6,
                       pf_tol=1e-12) for t in range(2)]
        runs.append((outs, h.get(U, w.maxlevel), h.get(D, w.maxlevel)))
        h.close()
    (o0, u0, d0), (o1, u1, d1) = runs
    assert [o[4] for o in o0] == [o[4] for o in o1]
    assert rel(u1, u0) < 1e-10 and rel(d1, d0) < 1e-10
    shapes = Hierarchy.tuned_shapes()
    assert shapes and all(s[3] in (2, 4, 8) and s[4] in (2, 4, 8, 16, 32) for s in shapes)
    assert {(33, 33, 33), (17, 17, 17), (9, 9, 9)} <= {s[:3] for s in shapes}
