"""TMA-staged finest applies against the cp.async-staged ones (GPU).

With hpc_set_tma_staging the finest-level operator applies (FP64, and the precision form's FP32)
bring each staged node row - three components on two planes - with one tensor copy into a
128-byte-aligned ring slot, the copy's x start rounded down to 16 bytes and the lanes reading from
the offset; out-of-range rows and columns arrive as zeros.  The element arithmetic sees the same
values as with the per-lane cp.async staging, so increments must agree bit for bit: step outputs and
the u, d, H fields, on cubic and anisotropic boxes (x extents that end mid-strip and strips whose
first column starts below zero), for the reference's FAS cycles and the precision form.
"""
import numpy as np
import pytest

from hpcrack_b200 import microstructure as ms
from hpcrack_b200.solver import Hierarchy, MECH_FAS, MECH_MIXED, U, D, H, precision_mg
from cases import load_workload

pytestmark = pytest.mark.gpu


def _run(w, solver, tma, steps):
    h = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start)
    h.set_tma_staging(tma)
    load_workload([h], w)
    mg_u = w.mg_u if solver == MECH_FAS else precision_mg(w.maxlevel, w.element_nb, w.mg_u[4])
    outs = [h.step(t, mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du, mech_tol=w.mech_tol,
                   pf_tol=w.pf_tol, mech_solver=solver) for t in range(steps)]
    fields = [h.get(f, w.maxlevel) for f in (U, D, H)]
    h.close()
    return outs, fields


@pytest.mark.parametrize("solver", [MECH_FAS, MECH_MIXED], ids=["fas", "mixed"])
@pytest.mark.parametrize("name", ["crack33", "box97x65x33", "parity65"])
def test_tma_staging_same_bits(name, solver):
    if name == "box97x65x33":
        w = ms.inclusion_workload(name, (97, 65, 33), 5, 0.25, None, 2)
    else:
        w = ms.make_workload(name)
    a = _run(w, solver, False, 2)
    b = _run(w, solver, True, 2)
    assert a[0] == b[0]
    for x, y in zip(a[1], b[1]):
        assert np.array_equal(x, y)
