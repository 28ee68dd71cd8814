"""Tensor-core element contraction of the precision form (GPU): with hpc_set_tensor_apply the FP32
V-cycle's element operator runs as two TF32 GEMMs per 128 elements on the tcgen05 tensor cores.
The flexible PCG around the V-cycle keeps its FP64 residual, so the solve meets the same FP64
tolerance; the TF32 operands (about 1e-3 relative) change the preconditioner slightly, hence the
number of outer iterations by a few at most and the solution by far less than the tolerance allows."""
import pytest

from hpcrack_b200 import microstructure as ms
from hpcrack_b200.solver import Hierarchy, MECH_MIXED, precision_mg
from cases import D, H, U, load_workload, rel

pytestmark = pytest.mark.gpu


def _solve(w, tc):
    h = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start)
    load_workload([h], w)
    h.set_tensor_apply(tc)
    mg = precision_mg(w.maxlevel, w.element_nb, 200)
    cy, _, fn = h.u_entire_fcg(mg, w.small_k, 1.0, 0, 0.0, mech_tol=1e-16, mixed=True)
    cy1, _, fn1 = h.u_entire_fcg(mg, w.small_k, 1.0, 1, fn, mech_tol=1e-16, mixed=True)
    r2 = h.initial_residual_u(w.maxlevel, w.small_k)
    u = h.get(U, w.maxlevel)
    h.close()
    return cy, cy1, r2 / fn1, u


@pytest.mark.parametrize("name", ["small33", "mid129"])
def test_tensor_apply_solve(name):
    w = ms.make_workload(name)
    cy_s, _, res_s, u_s = _solve(w, False)
    cy_t, cy1_t, res_t, u_t = _solve(w, True)
    assert res_t <= 1e-15, res_t  # the true FP64 residual, recomputed from scratch
    assert cy1_t == 0             # and the converged state passes the t >= 1 test at once
    assert abs(cy_t - cy_s) <= 3, (cy_t, cy_s)
    assert rel(u_t, u_s) < 1e-5


def test_tensor_apply_increments():
    w = ms.make_workload("small33")
    runs = []
    for tc in (False, True):
        h = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start)
        load_workload([h], w)
        h.set_tensor_apply(tc)
        for t in range(3):
            h.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du, mech_tol=1e-16,
                   pf_tol=1e-16, mech_solver=MECH_MIXED)
        runs.append([h.get(f, w.maxlevel) for f in (U, D, H)])
        h.close()
    for a, b in zip(*runs):
        assert rel(b, a) < 1e-5
