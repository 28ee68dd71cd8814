"""VTK output from the device (GPU): hpc_vtk_write's .vti / .pvti files are byte-identical to the
reference's write_total_de / write_total_u / write_total_H output (oracle/_ref) on the same data,
the write overlaps later work on the context without seeing it, and bad calls fail cleanly."""
import os

import numpy as np
import pytest

from cases import BULK, D, H, U, vtk_expected, vtk_paths
from hpcrack_b200 import lib as L
from hpcrack_b200 import microstructure as ms
from hpcrack_b200.solver import Hierarchy
from oracle import bindings as B

pytestmark = pytest.mark.gpu


def _pair(maxlevel, enb, x0):
    return Hierarchy(maxlevel, enb, x0=x0), B.RefOracle(maxlevel, enb, x0=x0)


@pytest.mark.skipif(not B.RefOracle.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("option,field,scale", [("S", D, 1.0), ("V", U, 0.3711), ("C", H, 1.0)])
@pytest.mark.parametrize("maxlevel,enb,x0", [(1, (4, 3, 2), (0.0, 0.0, 0.0)), (2, (3, 5, 2), (1.25, -2.5, 0.125)),
                                              (3, (8, 8, 8), (0.0, 0.0, 0.0))])
def test_vtk_matches_reference_writer(tmp_path, option, field, scale, maxlevel, enb, x0):
    h, ref = _pair(maxlevel, enb, x0)
    try:
        rng = np.random.default_rng(5)
        for level in (maxlevel, maxlevel - 1):
            n = h.n(level)
            vals = rng.standard_normal(3 * n if field == U else n) * 1e-3
            vals[::7] = 0.0
            h.set(field, level, vals)
            ref.set(field, level, vals)
            gdir, rdir = tmp_path / f"gpu{level}", tmp_path / f"ref{level}"
            for d in (gdir, rdir):
                os.makedirs(d / "Output")
            cwd = os.getcwd()
            os.chdir(gdir)
            try:
                h.vtk_write(option, field, level, "fld", "name", 3, scale=scale)
                h.vtk_wait()
            finally:
                os.chdir(cwd)
            ref.write_vtk(option, field, level, "fld", "name", 3, str(rdir), u_proportion=scale)
            for a, b in zip(vtk_paths(str(gdir), "fld", level, 3), vtk_paths(str(rdir), "fld", level, 3)):
                assert open(a, "rb").read() == open(b, "rb").read(), (a, level)
            # the float stream length exercises every tail of the 3-value groups across the cases
            dims = h.level_dims(level)[0]
            ev, ep = vtk_expected(option, vals, dims, (x0[0], x0[1], x0[2]), h.level_dims(level)[1], "fld", "name",
                                  level, 3, scale)
            assert open(vtk_paths(str(gdir), "fld", level, 3)[0], "rb").read() == ev
    finally:
        h.close()
        ref.close()


def test_vtk_write_overlaps_later_work(tmp_path):
    """The file holds the field as it was when the write was issued, although the context goes on
    (here: d is overwritten) before the write is waited for."""
    w = ms.make_workload("small17")
    h = Hierarchy(w.maxlevel, w.element_nb, x0=w.x_start)
    try:
        lv = w.maxlevel
        n = h.n(lv)
        d0 = np.linspace(0.0, 1.0, n)
        h.set(D, lv, d0)
        os.makedirs(tmp_path / "Output")
        cwd = os.getcwd()
        os.chdir(tmp_path)
        try:
            h.vtk_write("S", D, lv, "d", "d", 0)
            h.set(D, lv, np.zeros(n))
            h.vtk_write("S", D, lv, "z", "z", 1)  # waits for the first write, then starts its own
            h.vtk_wait()
        finally:
            os.chdir(cwd)
        dims, h3 = h.level_dims(lv)
        ev, _ = vtk_expected("S", d0, dims, w.x_start, h3, "d", "d", lv, 0)
        assert open(vtk_paths(str(tmp_path), "d", lv, 0)[0], "rb").read() == ev
        ez, _ = vtk_expected("S", np.zeros(n), dims, w.x_start, h3, "z", "z", lv, 1)
        assert open(vtk_paths(str(tmp_path), "z", lv, 1)[0], "rb").read() == ez
    finally:
        h.close()


def test_vtk_bad_calls(tmp_path):
    h = Hierarchy(1, (4, 3, 2))
    try:
        with pytest.raises(L.HpcError):
            h.vtk_write("VS", U, 1, "x", "x", 0)
        with pytest.raises(L.HpcError):
            h.vtk_write("S", U, 1, "x", "x", 0)  # a vector field for scalar output
        with pytest.raises(L.HpcError):
            h.vtk_write("V", BULK, 1, "x", "x", 0)
        with pytest.raises(L.HpcError):
            h.vtk_write("S", D, 5, "x", "x", 0)
        # no Output folder: the write fails when its thread opens the file
        cwd = os.getcwd()
        os.chdir(tmp_path)
        try:
            h.vtk_write("S", D, 1, "x", "x", 0)
            with pytest.raises(L.HpcError):
                h.vtk_wait()
            h.vtk_wait()  # nothing in flight any more
        finally:
            os.chdir(cwd)
    finally:
        h.close()
