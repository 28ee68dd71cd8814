"""History-dump format of the checkpoint files, pinned to the reference's own write_vector_3D /
read_vector_3D (write_read_history.cpp:18-86) compiled from its sources (oracle/_ref)."""
import os

import numpy as np
import pytest

from hpcrack_b200 import checkpoint as ck
from oracle import bindings as B

pytestmark = pytest.mark.skipif(not B.RefOracle.available(), reason="oracle/_ref not built")


def test_dump_path_matches_reference_pattern():
    assert ck.dump_path("run", "u", 7, 0) == os.path.join("run", "Time_step_data", "u_t_7_Proc_0.dat")


def test_reference_dump_reads_back(tmp_path):
    ref = B.RefOracle(1, (4, 3, 2))
    try:
        n = ref.n(1)
        rng = np.random.default_rng(3)
        for field, comp in ((B.U, 2), (B.H, 0), (B.D, 0)):
            a = rng.standard_normal(n)
            ref.set(field, 1, a[None].repeat(3, 0) if field == B.U else a)
            path = str(tmp_path / f"f{field}_t_0.dat")
            ref.write_vector_3d(field, 1, comp, path)
            assert "Write completed!" in ref.last_output()
            np.testing.assert_array_equal(ck.read_vector_3d(path, n), a)
    finally:
        ref.close()


def test_checkpoint_files_read_by_reference(tmp_path):
    ref = B.RefOracle(1, (4, 3, 2))
    try:
        n = ref.n(1)
        rng = np.random.default_rng(4)
        fields = {k: rng.standard_normal(n) for k in ("u", "v", "w", "H", "d", "d_old")}
        state = list(rng.standard_normal(6))
        paths = ck.write_checkpoint(str(tmp_path), 5, fields, state)
        assert len(paths) == 7
        for comp, key in enumerate(("u", "v", "w")):
            ref.read_vector_3d(B.U, 1, comp, ck.dump_path(str(tmp_path), key, 5))
            assert "Read completed!" in ref.last_output()
        ref.read_vector_3d(B.H, 1, 0, ck.dump_path(str(tmp_path), "H", 5))
        ref.read_vector_3d(B.D, 1, 0, ck.dump_path(str(tmp_path), "d", 5))
        u = ref.get(B.U, 1)
        for comp, key in enumerate(("u", "v", "w")):
            np.testing.assert_array_equal(u[comp], fields[key])
        np.testing.assert_array_equal(ref.get(B.H, 1), fields["H"])
        np.testing.assert_array_equal(ref.get(B.D, 1), fields["d"])
        back, st = ck.read_checkpoint(str(tmp_path), 5, n)
        assert st == state
        for k in fields:
            np.testing.assert_array_equal(back[k], fields[k])
        with pytest.raises(ValueError):
            ck.read_vector_3d(ck.dump_path(str(tmp_path), "u", 5), n + 1)
    finally:
        ref.close()
