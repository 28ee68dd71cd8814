"""GPU test of the allocation-free entry point hpc_dmax_noalloc (collected last on purpose).

Some callers of this library cannot allocate device memory while they run (their device memory
belongs to a pool allocator, or cudaMalloc's implicit synchronisation is not acceptable in their
loop).  hpc_dmax_noalloc serves them: it reduces caller-owned device arrays using only a fixed
__device__ scratch array.  Here it is called through the C ABI on device arrays the test owns, and
its output is checked against the context-based entry points hpc_delta_d_max / hpc_d_max on the
same values - on two calls in a row with different data, so that nothing left in the shared
scratch by the first call can leak into the second.  The maxima are exact, so the values must be
equal.
"""
import ctypes as C

import numpy as np
import pytest

from hpcrack_b200 import lib as L
from hpcrack_b200.solver import Hierarchy, D, DOLDF

pytestmark = pytest.mark.gpu


def _reference_values(hier, d, d_old):
    hier.set(D, hier.maxlevel, d)
    hier.set(DOLDF, hier.maxlevel, d_old)
    return hier.delta_d_max(), hier.d_max()


def test_noalloc_dmax_matches_context_entry_points():
    import torch

    lib = L.load()
    hier = Hierarchy(1, (8, 8, 8))  # finest level 17^3
    n = hier.n(1)
    rng = np.random.default_rng(5)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        d = rng.uniform(-0.5, 1.0, n) * (call + 1)
        d_old = d - rng.uniform(-0.2, 0.3, n)
        want_dd, want_dm = _reference_values(hier, d, d_old)
        td = torch.tensor(d, device="cuda")
        to = torch.tensor(d_old, device="cuda")
        rc = lib.hpc_dmax_noalloc(C.c_void_p(td.data_ptr()), C.c_void_p(to.data_ptr()), n,
                                  C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        L.check("hpc_dmax_noalloc", rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[0] == want_dd and got[1] == want_dm, (call, got, want_dd, want_dm)
    # a size of several hundred blocks with a ragged last block: the last block's combine loop
    # strides over more than 32 partials; the maxima are exact, so numpy gives the same values
    n_big = (1 << 20) + 12345
    d = rng.uniform(-0.5, 1.0, n_big)
    d_old = d - rng.uniform(-0.2, 0.3, n_big)
    d[n_big - 3] = 2.5  # the maximum sits in the partial last block
    td = torch.tensor(d, device="cuda")
    to = torch.tensor(d_old, device="cuda")
    for call in range(2):
        out.zero_()
        rc = lib.hpc_dmax_noalloc(C.c_void_p(td.data_ptr()), C.c_void_p(to.data_ptr()), n_big,
                                  C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        L.check("hpc_dmax_noalloc", rc)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[0] == max(0.0, float(np.max(d - d_old))) and got[1] == max(0.0, float(np.max(d))), (call, got)
    # sizes beyond the fixed scratch are refused with a clear error, before any launch
    rc = lib.hpc_dmax_noalloc(C.c_void_p(td.data_ptr()), C.c_void_p(to.data_ptr()), 134217729,
                              C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    assert rc == 1 and b"134217728" in lib.hpc_last_error()
    hier.close()
