"""CPU tests: the C-ABI library loads and exports every declared entry point, refuses to run
without a device (no CPU fallback), and the host-side logic (geometry, Dirichlet sets, image
generation, material table, maxlevel) matches the reference's."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from hpcrack_b200 import lib as L
from hpcrack_b200 import microstructure as ms
from oracle import bindings as B


def test_library_exports_every_declared_symbol():
    lib = L.load()
    declared = L.declared_symbols()
    assert len(declared) >= 45
    missing = [s for s in declared if not hasattr(lib, s)]
    assert missing == []
    # and the ctypes table covers them all
    assert sorted(L.SIGNATURES) == declared


def test_library_built_for_sm100a_only():
    """The build recipe compiles for sm_100a and nothing else (the runtime check of the built code is
    test_gpu_operators.py::test_binary_version_is_sm100)."""
    mk = open(os.path.join(os.path.dirname(L.LIB_PATH), "Makefile")).read()
    arch = [line for line in mk.splitlines() if line.startswith("ARCH")]
    assert arch == ["ARCH     := -gencode arch=compute_100a,code=sm_100a"], arch


def test_no_cpu_fallback_without_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except ImportError:
        pass
    lib = L.load()
    g = L.hpc_geometry(1, (C.c_int * 3)(8, 8, 8), (C.c_double * 3)(0, 0, 0), (C.c_int * 3)(0, 0, 0))
    h = C.c_void_p()
    rc = lib.hpc_create(C.byref(h), C.byref(g), 0)
    assert rc == 6 and not h.value  # HPC_ERR_NODEVICE
    assert b"no CPU path" in lib.hpc_last_error()
    v = C.c_int(0)
    assert lib.hpc_binary_version(C.byref(v)) == 6


def test_footprint_and_bad_geometry():
    lib = L.load()
    g = L.hpc_geometry(5, (C.c_int * 3)(8, 8, 8), (C.c_double * 3)(0, 0, 0), (C.c_int * 3)(0, 0, 0))
    b = C.c_size_t(0)
    assert lib.hpc_footprint(C.byref(g), C.byref(b)) == 0
    n = 260 * 257 * 257  # padded finest slots of 257^3
    # ~38 doubles per finest node allocated at creation (+1/7 for the coarse levels), plus what the
    # flexible forms, the Gauss-point moduli and a checkpoint allocate on first use (~55 more)
    assert 80 * 8 * n < b.value < 120 * 8 * n
    bad = L.hpc_geometry(-1, (C.c_int * 3)(8, 8, 8), (C.c_double * 3)(0, 0, 0), (C.c_int * 3)(0, 0, 0))
    assert lib.hpc_footprint(C.byref(bad), C.byref(b)) == 1


@pytest.mark.skipif(not B.RefOracle.available(), reason="reference oracle not built")
@pytest.mark.parametrize("ml,enb,x0", [(3, (2, 2, 2), (-16.0, -16.0, -16.0)), (2, (3, 5, 2), (0.5, -2.0, 7.0)),
                                       (1, (1, 1, 1), (0.0, 0.0, 0.0))])
def test_geometry_matches_reference_initialize(ml, enb, x0):
    ref = B.RefOracle(ml, enb, x0=x0)
    orc = B.COracle(ml, enb, x0=x0)
    for l in range(ml + 1):
        n3, h3, e3 = ref.level_info(l)
        assert n3 == orc.dims[l]
        assert n3 == tuple(e * 2 ** l + 1 for e in enb)
    ref.close()
    orc.close()


@pytest.mark.skipif(not B.RefOracle.available(), reason="reference oracle not built")
@pytest.mark.parametrize("enb", [(2, 2, 2), (3, 3, 3), (5, 2, 4)])
def test_dirichlet_sets_match_reference(enb):
    """Coordinate-equality node sets (boundary_conditions.cpp:20-68), including grids whose
    mid-point is not a node (odd element counts) so that a point constraint disappears."""
    ml = 2
    ref = B.RefOracle(ml, enb, x0=(-1.25, 3.0, 0.1))
    orc = B.COracle(ml, enb, x0=(-1.25, 3.0, 0.1))
    for l in range(ml + 1):
        n = ref.n(l)
        u = np.random.default_rng(l).standard_normal((3, n))
        for impl in (ref, orc):
            impl.set(B.U, l, u)
            impl.dirichlet_bd(l, B.U, 0.71)
        assert np.array_equal(ref.get(B.U, l), orc.get(B.U, l))
    ref.close()
    orc.close()


def test_sphere_image_deterministic_and_fractions():
    a = ms.sphere_image((65, 65, 65), 0, [ms.Phase(ms.INCLUSION_GRAY, 4, 8, count=12)])
    b = ms.sphere_image((65, 65, 65), 0, [ms.Phase(ms.INCLUSION_GRAY, 4, 8, count=12)])
    assert np.array_equal(a, b)
    assert set(np.unique(a)) <= {ms.MATRIX_GRAY, ms.INCLUSION_GRAY}
    c = ms.sphere_image((65, 65, 65), 3, [ms.Phase(ms.INCLUSION_GRAY, 4, 8, volume_fraction=0.2),
                                          ms.Phase(ms.PORE_GRAY, 2, 3, volume_fraction=0.03)])
    frac = (c == ms.INCLUSION_GRAY).mean()
    assert 0.14 < frac < 0.26
    assert (c == ms.PORE_GRAY).mean() > 0.01


def test_material_table_lands_on_phase_rows():
    """The integer-division gray interpolation (image_input.cpp:134-137) maps each label to its
    phase exactly with the breakpoint-pair table."""
    orc = B.COracle(0, (4, 1, 1))
    img = np.array([[[ms.MATRIX_GRAY, ms.PORE_GRAY, ms.INCLUSION_GRAY, ms.MATRIX_GRAY, ms.INCLUSION_GRAY]] * 2] * 2,
                   dtype=np.uint8)
    orc.image_material(img, (5, 2, 2), ms.material_table(), 1e-6)
    K = orc.get(B.BULK, 0)[:5]
    E = np.array([ms.MATRIX.E, ms.PORE.E, ms.INCLUSION.E, ms.MATRIX.E, ms.INCLUSION.E]) * 1e-6
    nu = np.array([ms.MATRIX.nu, ms.PORE.nu, ms.INCLUSION.nu, ms.MATRIX.nu, ms.INCLUSION.nu])
    assert np.allclose(K, E / (3 * (1 - 2 * nu)), rtol=1e-15)
    with pytest.raises(ValueError):
        bad = img.copy()
        bad[0, 0, 0] = 200
        orc.image_material(bad, (5, 2, 2), ([0, 84, 85, 169], [1, 1, 2, 2], [.2, .2, .2, .2], [1, 1, 1, 1]), 1e-6)
    orc.close()


@pytest.mark.skipif(not B.RefOracle.available(), reason="reference oracle not built")
def test_reference_input_path_matches_restatement():
    """The reference's raw-image + CSV reader (image_input.cpp, csv_reader.cpp) against the oracle's
    restatement, through files written by microstructure.write_inputs."""
    w = ms.make_workload("small17")
    ref = B.RefOracle(w.maxlevel, w.element_nb)
    orc = B.COracle(w.maxlevel, w.element_nb)
    with tempfile.TemporaryDirectory() as td:
        paths = ms.write_inputs(w, td)
        ref.input_total(td, paths["raw"], w.nodes, w.voxel_size)
        assert os.path.exists(paths["config"])
    orc.image_material(w.image, w.nodes, w.table(), w.voxel_size)
    for l in range(w.maxlevel + 1):
        for f in (B.BULK, B.G, B.GC):
            assert np.array_equal(ref.get(f, l), orc.get(f, l))
    ref.close()
    orc.close()


def test_maxlevel_rule():
    # main.cpp:52-68
    assert ms.maxlevel_for(129, 0, 4) == 5
    assert ms.maxlevel_for(65, 0, 8) == 3
    assert ms.maxlevel_for(257, 0, 8) == 5
    assert ms.maxlevel_for(9, 0, 8) == 0
    assert ms.maxlevel_for(17, 1, 8) == 0
