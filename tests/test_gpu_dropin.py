"""Drop-in test (GPU): the reference HPCrack program, and the same program with its hot-path
translation units replaced at link time by the C++ shims of hpcrack_b200/shim, run on the same
config.txt / Material_Property.csv / .raw inputs; their F_U.dat lines and per-increment history
dumps (Time_step_data/*.dat, the reference's own writer) and VTK files of d (Output/*.vti, *.pvti)
must agree.

Both programs run the reference's staggered loop until its stop test, so they are stopped after a
wall-clock budget and the increments both completed are compared.
"""
import base64
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from hpcrack_b200 import microstructure as ms

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "dropin", "_build")
PROG_REF = os.path.join(BUILD, "program_ref")
PROG_B200 = os.path.join(BUILD, "program_b200")


def _run(prog, workdir, seconds):
    with open(os.path.join(workdir, "stdout.txt"), "w") as out:
        try:
            subprocess.run([prog], cwd=workdir, stdout=out, stderr=subprocess.STDOUT, timeout=seconds)
        except subprocess.TimeoutExpired:
            pass


def _fu_lines(workdir):
    rows = {}
    path = os.path.join(workdir, "F_U.dat")
    if not os.path.exists(path):
        return rows
    for line in open(path):
        m = re.match(r"T= (\d+),U= (\S+) ,Fw= (\S+) ,deltaU= (\S+) ,delatad_max= (\S+)", line.strip())
        if m:
            rows[int(m.group(1))] = [float(m.group(i)) for i in range(2, 6)]
    return rows


def _vti_parts(data: bytes):
    head, rest = data.split(b'format="binary">\n', 1)
    payload, tail = rest.split(b"\n</DataArray>", 1)
    return head, payload, tail


def _vti_values(payload: bytes):
    n = int(np.frombuffer(base64.b64decode(payload[:8]), "<u4")[0])
    vals = np.frombuffer(base64.b64decode(payload[8:]), "<f4").astype(np.float64)
    assert vals.nbytes // 2 == n
    return vals


@pytest.mark.skipif(not (os.path.exists(PROG_REF) and os.path.exists(PROG_B200)),
                    reason="drop-in programs not built (make -C tests/dropin)")
def test_dropin_program_matches_reference_program():
    w = ms.make_workload("small17")
    root = tempfile.mkdtemp()
    try:
        dirs = {}
        for name in ("ref", "b200"):
            d = os.path.join(root, name)
            os.makedirs(d)
            # voxel 1e-5 m keeps the reaction above the reference's stop threshold for several increments
            w.voxel_size = 1e-5
            ms.write_inputs(w, d, extra={"outK": 0, "outG": 0, "outgc": 0, "outTdata": 1, "Tdatafrequence": 1})
            dirs[name] = d
        _run(PROG_B200, dirs["b200"], 45)
        _run(PROG_REF, dirs["ref"], 45)
        fr, fb = _fu_lines(dirs["ref"]), _fu_lines(dirs["b200"])
        common = sorted(set(fr) & set(fb))
        assert len(common) >= 2, (len(fr), len(fb), open(os.path.join(dirs["b200"], "stdout.txt")).read()[-2000:])
        for t in common:
            for a, b in zip(fr[t], fb[t]):
                assert abs(a - b) <= 1e-8 * max(abs(a), 1e-300) + 1e-300, (t, fr[t], fb[t])
            for field in ("u", "v", "w", "H", "d"):
                pa = os.path.join(dirs["ref"], "Time_step_data", f"{field}_t_{t}_Proc_0.dat")
                pb = os.path.join(dirs["b200"], "Time_step_data", f"{field}_t_{t}_Proc_0.dat")
                a, b = np.fromfile(pa), np.fromfile(pb)
                assert a.shape == b.shape
                na = np.linalg.norm(a)
                err = np.linalg.norm(a - b) / (na if na > 0 else 1.0)
                assert err < 1e-10, (t, field, err)
        # VTK output of d (write_total_de at t == 0 and once d_max >= 0.98): the reference's writer
        # in one program, the library's device encoder in the other; the same text, and Float32
        # values that agree to the rounding of values equal to 1e-10
        vtis = sorted(f for f in os.listdir(os.path.join(dirs["ref"], "Output")) if f.endswith("vti"))
        assert any(f.startswith("d_l_") and f.endswith("_t_0_Proc_0.vti") for f in vtis), vtis
        for f in vtis:
            t = int(re.search(r"_t_(\d+)", f).group(1))
            if t not in common or t == common[-1]:  # the last increment's write may have been cut off
                continue
            a = open(os.path.join(dirs["ref"], "Output", f), "rb").read()
            b = open(os.path.join(dirs["b200"], "Output", f), "rb").read()
            if f.endswith(".pvti"):
                assert a == b, f
                continue
            ha, pa, ta = _vti_parts(a)
            hb, pb, tb = _vti_parts(b)
            assert ha == hb and ta == tb, f
            va, vb = _vti_values(pa), _vti_values(pb)
            assert va.shape == vb.shape
            assert np.all(np.abs(va - vb) <= 1e-6 * np.maximum(np.abs(va), 1e-30)), f
    finally:
        shutil.rmtree(root, ignore_errors=True)
