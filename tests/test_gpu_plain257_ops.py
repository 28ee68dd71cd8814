"""The benchmarked 257^3 specimen's operators against the reference itself (GPU).

The benchmark times staggered increments of the 257^3 three-phase specimen (inclusions, pores at
E = 1 GPa, a d = 1 / H = H_crack pre-crack layer).  Whole increments of it are too slow for the
reference on a host (about ten minutes per V-cycle), so this test pins what the increments are made
of on the real fields of that specimen, once each, against the reference compiled from its own
sources (oracle/_ref):

* the raw-image + CSV input path: bulK, G, Gc on every level, bit for bit
  (image_input.cpp:120-282, the pore phase included);
* the regimes of a real displacement field: MP_choice on every element slot, exactly
  (material_selection.cpp:19-69);
* the element moduli: MP_all_element (material_selection.cpp:72-116) within 1e-13;
* the mechanical operator apply Internal_Force (mechanical_pcg.cpp:114-191) and its diagonal PreM_u,
  within 1e-12;
* the phase-field operator apply Fld (phase_field_pcg.cpp:61-103) on the pre-cracked d, within 1e-12;
* the history update strain_history (strain_history.cpp:162-210), within 1e-12.

The displacement is the library's own solution of the first increment's mechanical problem
(a few V-cycles), uploaded unchanged into the reference.  The reference runs on all host cores.
"""
import os
import tempfile

import numpy as np
import pytest

from oracle.bindings import RefOracle
from oracle import bindings as B
from hpcrack_b200 import microstructure as ms
from hpcrack_b200.solver import Hierarchy
from cases import rel

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not RefOracle.available(), reason="oracle/_ref/libhpcref.so not built")
def test_plain257_operators_against_reference():
    w = ms.make_workload("plain257")
    L = w.maxlevel
    Hc, dc = ms.precrack_fields(w)
    RefOracle._load().ref_set_threads(os.cpu_count() or 1)
    ref = RefOracle(L, w.element_nb, x0=w.x_start)
    with tempfile.TemporaryDirectory() as td:
        paths = ms.write_inputs(w, td)
        ref.input_total(td, paths["raw"], w.nodes, w.voxel_size)
    gpu = Hierarchy(L, w.element_nb, x0=w.x_start)
    gpu.image_material(w.image, w.nodes, w.table(), w.voxel_size)
    for impl in (ref, gpu):
        impl.set(B.H, L, Hc)
        impl.set(B.D, L, dc)
        impl.voigt_all_level(B.H)
    for l in range(L + 1):
        for f in (B.BULK, B.G, B.GC):
            assert np.array_equal(gpu.get(f, l), ref.get(f, l)), (l, f)

    # a displacement field of this specimen: the first increment's mechanical solve, a few V-cycles
    mg = tuple(w.mg_u[:4]) + (4,)
    gpu.u_entire(mg, w.small_k, 1.0, 0, 0.0)
    u = gpu.get(B.U, L)
    assert np.any(u != 0.0)
    ref.set(B.U, L, u)

    nx, ny, nz = w.nodes
    elem = np.zeros((nz, ny, nx), bool)
    elem[:-1, :-1, :-1] = True
    elem = elem.ravel()
    for impl in (ref, gpu):
        impl.mp_choice()
    ch_r, ch_g = ref.get_choice(L), gpu.get_choice(L)
    assert np.array_equal(ch_g[elem], ch_r[elem])
    assert len(np.unique(ch_r[elem])) >= 2  # the field exercises more than one regime

    for impl in (ref, gpu):
        impl.mp_all_element(w.small_k)
    assert rel(gpu.get(B.KE, L)[elem], ref.get(B.KE, L)[elem]) < 1e-13
    assert rel(gpu.get(B.GE, L)[elem], ref.get(B.GE, L)[elem]) < 1e-13

    for impl in (ref, gpu):
        impl.internal_force(L, B.U, B.RU, w.small_k)
    assert rel(gpu.get(B.RU, L), ref.get(B.RU, L)) < 1e-12
    for impl in (ref, gpu):
        impl.prem_u(L, B.RU, w.small_k)
    assert rel(gpu.get(B.RU, L), ref.get(B.RU, L)) < 1e-12

    for impl in (ref, gpu):
        impl.fld(L, B.D, B.FD, w.lc)
    assert rel(gpu.get(B.FD, L), ref.get(B.FD, L)) < 1e-12

    for impl in (ref, gpu):
        impl.strain_history(w.lc, w.ut0)
    H_r, H_g = ref.get(B.H, L), gpu.get(B.H, L)
    assert rel(H_g, H_r) < 1e-12
    outside = Hc == 0
    assert rel(H_g[outside & elem], H_r[outside & elem]) < 1e-12
    ref.close()
    gpu.close()
