"""Checkpoint / restart of the device-resident staggered loop (GPU).

A run of four increments is compared with a run restarted from the checkpoint written after the
second increment (through the reference's dump files): the restarted increments must reproduce the
uninterrupted ones bit for bit, since the checkpoint holds the loop's whole state.  The checkpoint
copy overlaps the next increment on the device, so the files are written only after that increment.
"""
import numpy as np
import pytest

from hpcrack_b200 import checkpoint as ck
from hpcrack_b200 import microstructure as ms
from hpcrack_b200.lib import HpcError
from hpcrack_b200.solver import Hierarchy
from cases import D, H, U, load_workload

pytestmark = pytest.mark.gpu


def _step(h, w, t):
    return h.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du, mech_tol=1e-6,
                  pf_tol=1e-12)


def test_restart_reproduces_uninterrupted_run(tmp_path):
    w = ms.make_workload("small17")
    L = w.maxlevel
    a = Hierarchy(L, w.element_nb, x0=w.x_start)
    load_workload([a], w)
    outs = []
    for t in range(4):
        outs.append(_step(a, w, t))
        if t == 1:
            a.checkpoint_begin(t)  # copy runs while increment 2 computes
        if t == 2:
            tck, fields, state = a.checkpoint_wait()
            assert tck == 1
            ck.write_checkpoint(str(tmp_path), tck, fields, state)
    final = {f: a.get(f, L) for f in (U, D, H)}
    a.close()

    b = Hierarchy(L, w.element_nb, x0=w.x_start)
    load_workload([b], w)  # material only; the loop state comes from the files
    fields, state = ck.read_checkpoint(str(tmp_path), 1, b.n(L))
    b.checkpoint_restore(fields, state)
    for t in (2, 3):
        o = _step(b, w, t)
        assert o == outs[t], (t, o, outs[t])
    for f, v in final.items():
        np.testing.assert_array_equal(b.get(f, L), v)
    b.close()


def test_checkpoint_wait_without_begin_fails():
    w = ms.make_workload("small17")
    h = Hierarchy(w.maxlevel, w.element_nb)
    with pytest.raises(HpcError, match="no checkpoint"):
        h.checkpoint_wait()
    h.close()
