"""VTK output format, pinned to the reference's own writers (vtk_output.cpp, compiled from its
sources in oracle/_ref): the files write_total_de / write_total_u / write_total_H produce are
byte-identical to the ones tests/cases.vtk_expected builds from the format's definition, which the
library's writer (hpc_vtk_write) is then held to on the GPU."""
import base64
import os

import numpy as np
import pytest

from cases import BULK, D, H, U, vtk_expected, vtk_paths
from oracle import bindings as B

pytestmark = pytest.mark.skipif(not B.RefOracle.available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("option,field,scale", [("S", D, 1.0), ("V", U, 0.3711), ("C", H, 1.0), ("S", BULK, 1.0)])
@pytest.mark.parametrize("enb,x0", [((4, 3, 2), (0.0, 0.0, 0.0)), ((3, 5, 2), (1.25, -2.5, 0.125))])
def test_reference_writer_matches_format(tmp_path, option, field, scale, enb, x0):
    ref = B.RefOracle(1, enb, x0=x0)
    try:
        level = 1
        n = ref.n(level)
        rng = np.random.default_rng(11)
        vals = rng.standard_normal(3 * n if field == U else n) * 1e-3
        ref.set(field, level, vals)
        os.makedirs(tmp_path / "Output")
        ref.write_vtk(option, field, level, "fld", "name", 4, str(tmp_path), u_proportion=scale)
        vti, pvti = vtk_paths(str(tmp_path), "fld", level, 4)
        dims, h3, _ = ref.level_info(level)
        box = ref.domain()
        ev, ep = vtk_expected(option, vals, dims, (box[0], box[2], box[4]), h3, "fld", "name", level, 4, scale)
        got = open(vti, "rb").read()
        assert got == ev
        assert open(pvti, "rb").read() == ep
        # and the payload decodes to the Float32 values
        body = got.split(b'format="binary">\n', 1)[1].split(b"\n</DataArray>", 1)[0]
        nbytes = np.frombuffer(base64.b64decode(body[:8]), "<u4")[0]
        data = np.frombuffer(base64.b64decode(body[8:]), "<f4")
        assert nbytes == data.nbytes
    finally:
        ref.close()
