"""Batched increments (hpc_batch_step) against one specimen at a time (hpc_step) (GPU).

A batch holds specimens of uneven, anisotropic sizes and different load histories; every specimen's
mechanical and phase-field solve runs as a device-driven loop inside one CUDA graph per batch.  The
loop bodies are the launches hpc_step makes, so each specimen's increments must agree bit for bit
with the same specimen run alone: step outputs (V-cycle and smoother counts, reaction, d maxima) and
the u, d, H fields.  Covered for the reference's FAS V-cycles, the flexible PCG and the precision
form, at t = 0 (forced first cycle, f_norm from the reactions) and later increments, with a batch
whose composition changes between calls (a specimen joins late, one leaves).
"""
import numpy as np
import pytest

from hpcrack_b200 import microstructure as ms
from hpcrack_b200.solver import (Batch, Hierarchy, MECH_FAS, MECH_FCG, MECH_MIXED, U, D, H, precision_mg,
                                 step_params)
from cases import load_workload

pytestmark = pytest.mark.gpu


def _specimens():
    return [ms.make_workload("small17"),
            ms.make_workload("crack33"),
            ms.inclusion_workload("box65x33x33", (65, 33, 33), 101, 0.2, None, 3),
            ms.inclusion_workload("box33x17x25", (33, 17, 25), 102, 0.3, None, 3)]


def _params(w, t, solver):
    mg_u = w.mg_u if solver == MECH_FAS else precision_mg(w.maxlevel, w.element_nb, w.mg_u[4])
    return step_params(t, mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du, mech_tol=w.mech_tol,
                       pf_tol=w.pf_tol, mech_solver=solver)


def _open(w):
    h = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start)
    load_workload([h], w)
    return h


def _fields(h, w):
    return [h.get(f, w.maxlevel) for f in (U, D, H)]


@pytest.mark.parametrize("solver", [MECH_FAS, MECH_FCG, MECH_MIXED], ids=["fas", "fcg", "mixed"])
def test_batch_matches_single_specimens(solver):
    ws = _specimens()
    steps = 2
    # alone
    alone = []
    for w in ws:
        h = _open(w)
        outs = [h.step(t, *_args(w, solver)) for t in range(steps)]
        alone.append((outs, _fields(h, w)))
        h.close()
    # together: crack33 joins one increment late, the others leave after their two increments
    schedule = [[0, 2, 3], [0, 1, 2, 3], [1]]
    hs = [_open(w) for w in ws]
    t_of = [0] * len(ws)
    outs = [[] for _ in ws]
    with Batch() as b:
        for idx in schedule:
            res = b.step([hs[i] for i in idx], [_params(ws[i], t_of[i], solver) for i in idx])
            for i, o in zip(idx, res):
                outs[i].append(o)
                t_of[i] += 1
    for i, w in enumerate(ws):
        n = len(outs[i])
        assert n == steps, (i, n)
        assert outs[i] == alone[i][0][:n], (w.name, outs[i], alone[i][0])
        for a, r in zip(_fields(hs[i], w), alone[i][1]):
            assert np.array_equal(a, r), w.name
        assert hs[i].launch_count() > 0
        hs[i].close()


def _args(w, solver):
    p = _params(w, 0, solver)
    mg_u = (p.mg_u.nu0, p.mg_u.nu1, p.mg_u.nu2, p.mg_u.gamma, p.mg_u.ncy)
    return (mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, w.ut0, w.du, 1.5e-3, w.mech_tol, w.pf_tol, solver)
