"""One specimen split along z over slab ranks against the same specimen in one context (GPU).

The ranks are slab contexts of this process on one device, one host thread each, joined by the
library's in-process transport (SlabGroup); the decomposition, ghost exchanges and reductions are the
ones a multi-GPU run makes over NCCL.  The coarsest level is either gathered and solved redundantly by
the one-block solver (the default, as the whole specimen solves it) or solved by the distributed
per-iteration smoother (hpc_set_fused_coarsest(0) on both sides), so the two differ only in the order
of the reductions' sums: operators and transfers agree to rounding, staggered increments within 1e-10
with equal V-cycle counts (on pre-cracked specimens from the second increment on within the spreads of
tests/cases.py).  A one-rank slab over NCCL reproduces the whole specimen bit for bit.
"""
import os
import time

import numpy as np
import pytest

from hpcrack_b200 import lib as L
from hpcrack_b200 import microstructure as ms
from hpcrack_b200.slab import SlabGroup, join_nccl, nccl_unique_id
from hpcrack_b200.solver import MECH_FCG, MECH_MIXED, Batch, Hierarchy, precision_mg, step_params
from cases import (BULK, CRACK_CYCLE_SLACK, CRACK_F_TOL, CRACK_U_TOL, D, FD, FU, GC, G, H, R, RU, U, UOLD,
                   load_random, load_workload, rel)

pytestmark = pytest.mark.gpu


def _whole(maxlevel, enb, x0=(0.0, 0.0, 0.0), fused=False):
    h = Hierarchy(maxlevel, enb, x0=x0)
    h.set_fused_coarsest(fused)
    return h


@pytest.mark.parametrize("nranks", [2, 3])
def test_slab_operators_transfers_and_reductions_match_the_whole_specimen(nranks):
    ml, enb = 2, (2, 3, 4)  # 9 x 13 x 17 finest nodes; 3 ranks: 2 / 3 / 4 coarsest planes, with ghosts
    whole = _whole(ml, enb)
    split = SlabGroup(ml, enb, nranks)
    split.set_fused_coarsest(False)
    try:
        load_random([whole, split], ml, enb, seed=3)
        for l in range(ml + 1):
            for impl in (whole, split):
                impl.internal_force(l, U, RU, 1e-5)
            assert rel(split.get(RU, l), whole.get(RU, l)) < 1e-14, l
            for impl in (whole, split):
                impl.prem_u(l, RU, 1e-5)
            assert rel(split.get(RU, l), whole.get(RU, l)) < 1e-14, l
            for impl in (whole, split):
                impl.fld(l, D, FD, 2.0)
            assert rel(split.get(FD, l), whole.get(FD, l)) < 1e-14, l
            # reductions over owned planes, combined over the ranks
            a, b = whole.initial_residual_u(l, 1e-5), split.initial_residual_u(l, 1e-5)
            assert abs(a - b) <= 1e-13 * abs(a), (l, a, b)
            a, b = whole.initial_residual_d(l, 2.0), split.initial_residual_d(l, 2.0)
            assert abs(a - b) <= 1e-13 * abs(a), (l, a, b)
        for lf in range(1, ml + 1):
            for comp in range(3):
                for impl in (whole, split):
                    impl.solution_injection(U, comp, lf)
                assert np.array_equal(split.get(U, lf - 1)[comp], whole.get(U, lf - 1)[comp]), (lf, comp)
                for impl in (whole, split):
                    impl.coarsen_f_standard(RU, FU, UOLD, comp, lf)
                assert rel(split.get(RU, lf - 1)[comp], whole.get(RU, lf - 1)[comp]) < 1e-14, (lf, comp)
                for impl in (whole, split):
                    impl.refine_standard(U, RU, UOLD, comp, lf)
                assert rel(split.get(U, lf)[comp], whole.get(U, lf)[comp]) < 1e-14, (lf, comp)
        for impl in (whole, split):
            impl.vr_all_level(BULK)
            impl.coarse_vr(G)
        for l in range(ml + 1):
            assert rel(split.get(BULK, l), whole.get(BULK, l)) < 1e-14, l
            assert rel(split.get(G, l), whole.get(G, l)) < 1e-14, l
        # one smoother call of pcg_u (direction exchanged after every update)
        for impl in (whole, split):
            impl.prem_u(ml, RU, 1e-5)
        _, fw = whole.pcg_u(ml, 1e-5, 1.0, 6, 1, 1.0)
        _, fs = split.pcg_u(ml, 1e-5, 1.0, 6, 1, 1.0)
        assert rel(split.get(U, ml), whole.get(U, ml)) < 1e-12
        assert split.d_max() == whole.d_max() and split.delta_d_max() == whole.delta_d_max()
    finally:
        whole.close()
        split.close()


CASES = [("small33", 2, 3, "gathered"), ("crack33", 2, 3, "gathered"), ("crack33", 3, 2, "gathered"),
         ("crack33", 3, 2, "distributed"), ("box65x33x33", 4, 2, "distributed")]


def _workload(name):
    if name.startswith("box"):
        return ms.inclusion_workload(name, (65, 33, 33), 101, 0.2, None, 2)
    return ms.make_workload(name)


@pytest.mark.parametrize("name,nranks,steps,coarsest", CASES, ids=[f"{n}-{r}ranks-{c}" for n, r, _, c in CASES])
def test_slab_increments_match_the_whole_specimen(name, nranks, steps, coarsest):
    w = _workload(name)
    fused = coarsest == "gathered"
    whole = _whole(w.maxlevel, w.element_nb, w.x_start, fused=fused)
    split = SlabGroup(w.maxlevel, w.element_nb, nranks, x0=w.x_start)
    split.set_fused_coarsest(fused)
    try:
        load_workload([whole, split], w)
        Lf = w.maxlevel
        for l in range(Lf + 1):
            for f in (BULK, G, GC):
                assert rel(split.get(f, l), whole.get(f, l)) == 0.0, (l, f)
        assert rel(split.get(H, 0), whole.get(H, 0)) < 1e-15
        cracked = w.crack is not None
        kw = dict(ut0=w.ut0, dU=w.du, mech_tol=w.mech_tol, pf_tol=w.pf_tol)
        for t in range(steps):
            ow = whole.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, **kw)
            osl = split.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, **kw)
            assert ow[5] == osl[5] and ow[7] == osl[7], (t, ow, osl)
            if t == 0 or not cracked:
                assert ow[4] == osl[4] and ow[6] == osl[6], (t, ow, osl)
                assert rel(split.get(U, Lf), whole.get(U, Lf)) < 1e-10, t
                assert abs(ow[1] - osl[1]) <= 1e-10 * abs(ow[1]), (t, ow, osl)
            else:
                assert abs(ow[4] - osl[4]) <= CRACK_CYCLE_SLACK, (t, ow, osl)
                assert rel(split.get(U, Lf), whole.get(U, Lf)) < CRACK_U_TOL[w.mech_tol], t
                assert abs(ow[1] - osl[1]) <= CRACK_F_TOL[w.mech_tol] * abs(ow[1]), t
            assert rel(split.get(D, Lf), whole.get(D, Lf)) < 1e-10, t
            assert rel(split.get(H, Lf), whole.get(H, Lf)) < 1e-10, t
            assert abs(ow[2] - osl[2]) <= 1e-12 and abs(ow[3] - osl[3]) <= 1e-12 * max(abs(ow[3]), 1.0), t
        if cracked:
            assert ow[5] >= 1  # the phase field moved
    finally:
        whole.close()
        split.close()


@pytest.mark.parametrize("name,solver", [("small33", MECH_MIXED), ("crack33", MECH_MIXED), ("small33", MECH_FCG)],
                         ids=["small33-mixed", "crack33-mixed", "small33-fcg"])
def test_slab_flexible_forms_match_the_whole_specimen(name, solver):
    """The flexible PCG (FP64 V-cycle, or the precision form's FP32 V-cycle) on 2 slab ranks against the
    whole specimen: both solve each increment to |r|/|f| <= 1e-8, the FP32 cycle amplifies the
    different order of the sums, so the bar is the one the forms meet against each other (1e-6)."""
    w = ms.make_workload(name)
    mg_u = precision_mg(w.maxlevel, w.element_nb, w.mg_u[4])
    whole = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start)
    split = SlabGroup(w.maxlevel, w.element_nb, 2, x0=w.x_start)
    try:
        load_workload([whole, split], w)
        Lf = w.maxlevel
        kw = dict(ut0=w.ut0, dU=w.du, mech_tol=w.mech_tol, pf_tol=w.pf_tol, mech_solver=solver)
        for t in range(2):
            ow = whole.step(t, mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, **kw)
            osl = split.step(t, mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, **kw)
            assert abs(ow[4] - osl[4]) <= 1 and abs(ow[5] - osl[5]) <= 1, (t, ow, osl)
            for f in (U, D, H):
                assert rel(split.get(f, Lf), whole.get(f, Lf)) < 1e-6, (t, f)
            assert abs(ow[1] - osl[1]) <= 1e-6 * abs(ow[1]), (t, ow, osl)
    finally:
        whole.close()
        split.close()


def test_one_rank_slab_over_nccl_reproduces_the_whole_specimen():
    os.environ.setdefault("NCCL_SOCKET_IFNAME", "lo")
    w = ms.make_workload("crack33")
    whole = _whole(w.maxlevel, w.element_nb, w.x_start, fused=True)
    one = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start, slab=(1, 0))
    try:
        join_nccl(one, nccl_unique_id())
        load_workload([whole, one], w)
        kw = dict(ut0=w.ut0, dU=w.du, mech_tol=w.mech_tol, pf_tol=w.pf_tol)
        for t in range(2):
            ow = whole.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, **kw)
            oo = one.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, **kw)
            assert ow == oo, (t, ow, oo)
        for f in (U, D, H):
            assert np.array_equal(one.get(f, w.maxlevel), whole.get(f, w.maxlevel)), f
    finally:
        whole.close()
        one.close()


def test_slab_refusals_and_abort():
    w = ms.make_workload("small17")
    split = SlabGroup(w.maxlevel, w.element_nb, 2, x0=w.x_start)
    try:
        load_workload([split], w)
        with pytest.raises(L.HpcError):
            split.set_autotune(True)
        p = step_params(0, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du)
        with Batch() as b, pytest.raises(L.HpcError):
            b.step([split.ranks[0]], [p])

        # a rank that fails before a collective step ends the other rank's wait (no hang, an error)
        def fn(h):
            if h.slab[1] == 1:
                raise RuntimeError("rank 1 failed")
            return h.initial_residual_u(w.maxlevel, w.small_k)

        t0 = time.time()
        with pytest.raises(RuntimeError, match="rank 1 failed"):
            split.run(fn)
        assert time.time() - t0 < 60
    finally:
        split.close()


def test_split_cracked_specimen_matches_the_oracle():
    """crack33 (the benchmarked recipe: pores, inclusions, pre-crack) split over 3 ranks against the C
    oracle, which the reference's own goldens pin: the first increment within 1e-10 on u, d, H with
    equal V-cycle and finest-iteration counts, the second within the reference's own run-to-run
    spread on u and the reaction (tests/cases.py), d and H within 1e-10."""
    from oracle.bindings import COracle

    w = ms.make_workload("crack33")
    split = SlabGroup(w.maxlevel, w.element_nb, 3, x0=w.x_start)
    orc = COracle(w.maxlevel, w.element_nb, x0=w.x_start)
    try:
        load_workload([split, orc], w)
        Lf = w.maxlevel
        kw = dict(ut0=w.ut0, dU=w.du, mech_tol=w.mech_tol, pf_tol=w.pf_tol)
        for t in range(2):
            og = split.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, **kw)
            oo = orc.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, **kw)
            assert og[5] == oo[5] and og[7] == oo[7], (t, og, oo)
            if t == 0:
                assert og[4] == oo[4] and og[6] == oo[6], (t, og, oo)
                assert rel(split.get(U, Lf), orc.get(U, Lf)) < 1e-10
                assert abs(og[1] - oo[1]) <= 1e-10 * abs(oo[1])
            else:
                assert abs(og[4] - oo[4]) <= CRACK_CYCLE_SLACK, (t, og, oo)
                assert rel(split.get(U, Lf), orc.get(U, Lf)) < CRACK_U_TOL[w.mech_tol], t
                assert abs(og[1] - oo[1]) <= CRACK_F_TOL[w.mech_tol] * abs(oo[1]), t
            assert rel(split.get(D, Lf), orc.get(D, Lf)) < 1e-10, t
            assert rel(split.get(H, Lf), orc.get(H, Lf)) < 1e-10, t
    finally:
        split.close()
        orc.close()
