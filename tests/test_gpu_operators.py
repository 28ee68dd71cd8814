"""Parity of the CUDA operators with the C oracle on seeded random fields (GPU).

FP64 throughout; the CUDA kernels sum-factorise the Q1 element algebra and use FMA, so they
differ from the oracle only by rounding: relative L2 tolerance 1e-12 on operator outputs.
"""
import numpy as np
import pytest

from oracle.bindings import COracle
from hpcrack_b200.solver import Hierarchy
from cases import BULK, G, GC, D, H, FD, KE, GE, R, U, FU, RU, UOLD, load_random, rel

pytestmark = pytest.mark.gpu
TOL = 1e-12

GEOMS = [
    (2, (2, 2, 2), (0, 0, 0)),     # 9^3 finest, 3^3 coarsest
    (2, (4, 3, 5), (0, 0, 0)),     # anisotropic 17 x 13 x 21
    (1, (8, 2, 3), (0, 0, 0)),     # 17 x 5 x 7 (nx > ny: the MP_choice loop-bound quirk matters)
    (1, (2, 7, 3), (0, 0, 0)),     # 5 x 15 x 7 (ny > nx)
    (0, (30, 3, 2), (0, 0, 0)),    # single level, 31 x 4 x 3: strips wider than a warp
    # an image ROI start (input_setting, image_input.cpp:21-27) makes hx, hy, hz differ: the kernels
    # without the isotropic 1/h^2 folding
    (1, (4, 3, 2), (1, 2, 0)),     # 9 x 7 x 5, h = (2.25, 2.67, 2) on level 0
]


@pytest.fixture(params=GEOMS, ids=lambda g: f"L{g[0]}-{g[1][0]}x{g[1][1]}x{g[1][2]}-roi{g[2][0]}{g[2][1]}{g[2][2]}")
def pair(request):
    ml, enb, roi = request.param
    x0 = (-3.0, 1.5, -7.0)
    gpu = Hierarchy(ml, enb, x0=x0, roi=roi)
    orc = COracle(ml, enb, x0=x0, roi=roi)
    load_random([gpu, orc], ml, enb, seed=123)
    yield ml, gpu, orc
    gpu.close()
    orc.close()


def test_internal_force(pair):
    ml, gpu, orc = pair
    for l in range(ml + 1):
        gpu.internal_force(l, U, RU, 1e-5)
        orc.internal_force(l, U, RU, 1e-5)
        assert rel(gpu.get(RU, l), orc.get(RU, l)) < TOL, l


def test_prem_u(pair):
    ml, gpu, orc = pair
    for l in range(ml + 1):
        gpu.prem_u(l, RU, 1e-5)
        orc.prem_u(l, RU, 1e-5)
        assert rel(gpu.get(RU, l), orc.get(RU, l)) < TOL, l


def test_fld_and_diag(pair):
    ml, gpu, orc = pair
    for l in range(ml + 1):
        gpu.fld(l, D, FD, 2.0)
        orc.fld(l, D, FD, 2.0)
        assert rel(gpu.get(FD, l), orc.get(FD, l)) < TOL, l
        gpu.precondition_m(l, R, 2.0)
        orc.precondition_m(l, R, 2.0)
        assert rel(gpu.get(R, l), orc.get(R, l)) < TOL, l


def test_transfers(pair):
    ml, gpu, orc = pair
    for lf in range(1, ml + 1):
        for comp in range(3):
            for impl in (gpu, orc):
                impl.solution_injection(U, comp, lf)
            assert rel(gpu.get(U, lf - 1)[comp], orc.get(U, lf - 1)[comp]) == 0.0
            for impl in (gpu, orc):
                impl.coarsen_f_standard(RU, FU, UOLD, comp, lf)
            assert rel(gpu.get(RU, lf - 1)[comp], orc.get(RU, lf - 1)[comp]) < 1e-14
            for impl in (gpu, orc):
                impl.refine_standard(FU, U, UOLD, comp, lf)
            assert rel(gpu.get(FU, lf)[comp], orc.get(FU, lf)[comp]) < 1e-14


def test_boundary_conditions(pair):
    ml, gpu, orc = pair
    for l in range(ml + 1):
        for impl in (gpu, orc):
            impl.dirichlet_bd(l, U, 0.37)
        assert np.array_equal(gpu.get(U, l), orc.get(U, l))
        for impl in (gpu, orc):
            impl.dirichlet_force(l, FU, U)
        assert np.array_equal(gpu.get(FU, l), orc.get(FU, l))
        for impl in (gpu, orc):
            impl.dirichlet_residual(l, FU)
        assert np.array_equal(gpu.get(FU, l), orc.get(FU, l))


def test_material_selection(pair):
    ml, gpu, orc = pair
    for quirk in (True, False):
        gpu.set_choice_quirk(quirk)
        orc.set_choice_quirk(quirk)
        gpu.mp_choice()
        orc.mp_choice()
        L = ml
        nx, ny, nz = gpu.dims[L]
        elem = np.zeros((nz, ny, nx), bool)
        elem[:-1, :-1, :-1] = True
        elem = elem.ravel()
        cg, co = gpu.get_choice(L), orc.get_choice(L)
        assert np.array_equal(cg[elem], co[elem]), quirk
        gpu.mp_all_element(1e-5)
        orc.mp_all_element(1e-5)
        assert rel(gpu.get(KE, L)[elem], orc.get(KE, L)[elem]) < TOL
        assert rel(gpu.get(GE, L)[elem], orc.get(GE, L)[elem]) < TOL


def test_coarse_material(pair):
    ml, gpu, orc = pair
    for impl in (gpu, orc):
        impl.vr_all_level(KE)
        impl.voigt_all_level(H)
        impl.coarse_vr(GC)
    for l in range(ml + 1):
        assert rel(gpu.get(KE, l), orc.get(KE, l)) < 1e-14
        assert rel(gpu.get(H, l), orc.get(H, l)) < 1e-14
        assert rel(gpu.get(GC, l), orc.get(GC, l)) < 1e-14


def test_history_rhs_reductions(pair):
    ml, gpu, orc = pair
    for impl in (gpu, orc):
        impl.strain_history(2.0, 3.5)
    assert rel(gpu.get(H, ml), orc.get(H, ml)) < 1e-12
    for l in range(ml + 1):
        for impl in (gpu, orc):
            impl.fd_h(l)
        # fd_h sums in the reference's scatter order with uncontracted IEEE operations
        assert rel(gpu.get(FD, l), orc.get(FD, l)) < 1e-15, (l, rel(gpu.get(FD, l), orc.get(FD, l)))
    assert gpu.d_max() == orc.d_max()
    assert gpu.delta_d_max() == orc.delta_d_max()
    assert abs(gpu.externe_force_sum() - orc.externe_force_sum()) <= 1e-12 * max(1.0, abs(orc.externe_force_sum()))
    ug, uo = gpu.U_e(2.0), orc.U_e(2.0)
    assert abs(ug - uo) <= 1e-12 * abs(uo)


def test_initial_crack(pair):
    ml, gpu, orc = pair
    for l in range(ml + 1):
        for impl in (gpu, orc):
            impl.initial_crack(7.5, l)
        assert np.array_equal(gpu.get(H, l), orc.get(H, l))


def test_binary_version_is_sm100():
    """The runtime reports the library's kernels as built for compute capability 10.0 (sm_100a)."""
    import ctypes as C
    from hpcrack_b200 import lib as L
    v = C.c_int(0)
    L.check("hpc_binary_version", L.load().hpc_binary_version(C.byref(v)))
    assert v.value == 100, v.value
