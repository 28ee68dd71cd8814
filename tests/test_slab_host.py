"""CPU tests of the z-slab decomposition (one specimen split along z over ranks).

1. hpc_slab_level (host only) against the reference's own per-rank formulas, restated here:
   initialize's node counts (initialization.cpp:50-72 for the coarsest level, :92-125 for the finer
   ones), get_coordinate (boundary_conditions.cpp:13-18) and realdomain (realdomain.h:17-40).
2. The properties the library's kernels rely on: the owned planes tile the specimen in rank order on
   every level, each ghost plane is a neighbour's edge plane, coarse plane kc lies on fine plane
   2 kc + zsh with zsh in {0, -1}, owned coarse nodes fall on owned fine nodes.
3. A world-size-2 gloo run of the exchange schedule the library follows (slab.cu): Jacobi-PCG with a
   7-point operator on two slabs, the direction's ghost planes exchanged after every direction update
   (plane 1 to the rank below, plane nz-2 to the rank above) and the dot products summed over owned
   planes and all-reduced, against the same PCG on the whole grid.
"""
import os
import socket

import numpy as np
import pytest

from hpcrack_b200 import lib as L
from hpcrack_b200.solver import slab_level


# ---------------------------------------------------------------- the reference's formulas
def ref_nbcolo(kk0, npz, coord, maxlevel):
    """nbcoloz per level (initialization.cpp:50-72, :92-125)."""
    q = (kk0 + 1) // npz
    if npz == 1:
        n = kk0 + 1
    else:
        n = q + 2
        if coord == 0:
            n = q + 1
        if coord == npz - 1:
            n = q + (kk0 + 1) % npz + 1
    out = []
    for _ in range(maxlevel + 1):
        out.append(n)
        if npz == 1 or coord == 0:
            n = 2 * (n - 1) + 1
        elif coord == npz - 1:
            n = 2 * (n - 1)
        else:
            n = 2 * (n - 2) + 2
    return out


def ref_global_index(coord, npz, total, nbcolo, index):
    """get_coordinate (boundary_conditions.cpp:13-18) with origin 0 and spacing 1."""
    if coord == 0:
        return index
    if coord == npz - 1:
        return total - nbcolo + 1 + index
    return coord * (nbcolo - 2) + index - 1


def ref_realdomain(n, coord, npz):
    """realdomain (realdomain.h:17-40) along one axis: [lo, hi)."""
    lo, hi = 0, n
    if npz > 1:
        if coord == 0:
            hi = n - 1
        elif coord == npz - 1:
            lo = 1
        else:
            lo, hi = 1, n - 1
    return lo, hi


CASES = [(kk0, ml, npz) for kk0 in range(1, 21) for ml in range(0, 5) for npz in range(1, 9)]


@pytest.mark.parametrize("kk0,maxlevel,npz", CASES)
def test_slab_plan_matches_reference_decomposition(kk0, maxlevel, npz):
    enb = (2, 3, kk0)
    if (kk0 + 1) // npz < 1:
        with pytest.raises(L.HpcError):
            slab_level(maxlevel, enb, npz, 0, 0)
        return
    plans = [[slab_level(maxlevel, enb, npz, r, l) for l in range(maxlevel + 1)] for r in range(npz)]
    for r in range(npz):
        ns = ref_nbcolo(kk0, npz, r, maxlevel)
        for l in range(maxlevel + 1):
            nz, zb, lo, hi = plans[r][l]
            assert nz == ns[l], (r, l)
            assert zb == ref_global_index(r, npz, kk0 << l, nz, 0), (r, l)
            assert (lo, hi) == ref_realdomain(nz, r, npz), (r, l)
    for l in range(maxlevel + 1):
        nzg = (kk0 << l) + 1
        # owned planes tile [0, nzg) in rank order
        cur = 0
        for r in range(npz):
            nz, zb, lo, hi = plans[r][l]
            assert zb + lo == cur and hi > lo
            cur = zb + hi
            # ghosts: one plane beyond the owned ones towards each neighbour, nothing else
            assert lo == (1 if r > 0 else 0) and hi == (nz - 1 if r < npz - 1 else nz)
            if r > 0:  # my plane 0 is the rank below's last owned plane (its plane nz-2)
                nzb, zbb, _, hib = plans[r - 1][l]
                assert zb == zbb + hib - 1 and hib == nzb - 1
            if r < npz - 1:  # my plane nz-1 is the rank above's first owned plane (its plane 1)
                assert zb + nz - 1 == plans[r + 1][l][1] + 1
        assert cur == nzg
        if l < maxlevel:
            for r in range(npz):
                nzc, zbc, loc, hic = plans[r][l]
                nzf, zbf, lof, hif = plans[r][l + 1]
                zsh = 2 * zbc - zbf
                assert zsh in (0, -1) and (zsh == 0) == (r == 0 or npz == 1)
                for kc in range(loc, hic):  # owned coarse nodes land on owned fine nodes
                    assert lof <= 2 * kc + zsh < hif
                assert 2 * (nzc - 1) + zsh <= nzf - 1  # every coarse plane's fine plane exists (or is < 0)


def test_every_declared_slab_entry_point_is_exported():
    lib = L.load()
    for name in ("hpc_slab_level", "hpc_create_slab", "hpc_slab_group_create", "hpc_slab_group_join",
                 "hpc_slab_group_abort", "hpc_slab_group_destroy", "hpc_nccl_unique_id", "hpc_slab_join_nccl"):
        assert hasattr(lib, name), name


# ---------------------------------------------------------------- two ranks over gloo
torch = pytest.importorskip("torch")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _apply(u):
    """7-point operator 6u - sum of the neighbours, zero outside the array (z, y, x axes)."""
    out = 6.0 * u
    for ax in range(3):
        out[tuple(slice(1, None) if a == ax else slice(None) for a in range(3))] -= \
            u[tuple(slice(None, -1) if a == ax else slice(None) for a in range(3))]
        out[tuple(slice(None, -1) if a == ax else slice(None) for a in range(3))] -= \
            u[tuple(slice(1, None) if a == ax else slice(None) for a in range(3))]
    return out


def _pcg(f, iters, dot, exchange):
    """Restarted Jacobi-PCG of mechanical_pcg.cpp:268-321 (beta = 0 first) on one array."""
    u = np.zeros_like(f)
    r = f - _apply(u)
    p = np.zeros_like(f)
    rz_old = None
    for i in range(iters):
        z = r / 6.0
        rz = dot(r, z)
        p = z if i == 0 else z + (rz / rz_old) * p
        exchange(p)
        w = _apply(p)
        alpha = rz / dot(p, w)
        u += alpha * p
        r -= alpha * w
        rz_old = rz
    return u


GEOM = dict(maxlevel=2, enb=(2, 2, 3))


def _global_f():
    nzg = (GEOM["enb"][2] << GEOM["maxlevel"]) + 1
    ny = (GEOM["enb"][1] << GEOM["maxlevel"]) + 1
    nx = (GEOM["enb"][0] << GEOM["maxlevel"]) + 1
    return np.random.default_rng(5).standard_normal((nzg, ny, nx))


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        nz, zb, lo, hi = slab_level(GEOM["maxlevel"], GEOM["enb"], world, rank, GEOM["maxlevel"])
        fg = _global_f()
        f = fg[zb:zb + nz].copy()
        f[:lo] = 0.0  # a rank's right-hand side only matters on its owned planes
        f[hi:] = 0.0

        def dot(a, b):
            t = torch.tensor([float(np.sum(a[lo:hi] * b[lo:hi]))], dtype=torch.float64)
            dist.all_reduce(t)
            return float(t[0])

        def exchange(p):
            reqs, bufs = [], []
            if rank > 0:
                reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(p[1])), rank - 1))
                bufs.append((0, torch.empty(p[0].shape, dtype=torch.float64)))
                reqs.append(dist.irecv(bufs[-1][1], rank - 1))
            if rank < world - 1:
                reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(p[nz - 2])), rank + 1))
                bufs.append((nz - 1, torch.empty(p[0].shape, dtype=torch.float64)))
                reqs.append(dist.irecv(bufs[-1][1], rank + 1))
            for rq in reqs:
                rq.wait()
            for k, b in bufs:
                p[k] = b.numpy()

        u = _pcg(f, 12, dot, exchange)
        q.put((rank, zb, lo, hi, u[lo:hi].copy()))
    finally:
        dist.destroy_process_group()


def test_two_slab_ranks_reproduce_the_whole_grid_pcg():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    fg = _global_f()
    whole = _pcg(fg, 12, lambda a, b: float(np.sum(a * b)), lambda p: None)
    split = np.concatenate([u for _, _, _, _, u in res], axis=0)
    assert [zb + lo for _, zb, lo, _, _ in res] == [0, res[0][1] + res[0][3]]
    assert split.shape == whole.shape
    err = np.linalg.norm(split - whole) / np.linalg.norm(whole)
    assert err < 1e-12, err


# ---------------------------------------------------------------- whole-specimen arrays <-> ranks
class _FakeRank:
    """Stands in for a slab context: its plan and local arrays (no device)."""

    def __init__(self, maxlevel, enb, nranks, rank):
        self.plans = [slab_level(maxlevel, enb, nranks, rank, l) for l in range(maxlevel + 1)]
        self.dims = [((enb[0] << l) + 1, (enb[1] << l) + 1, self.plans[l][0]) for l in range(maxlevel + 1)]
        self.slab = (nranks, rank)
        self.store = {}

    def set(self, field, level, arr):  # the layout Hierarchy.set takes: flat, or (3, n) for vectors
        from hpcrack_b200.solver import VECTOR_FIELDS
        a = np.array(arr, dtype=np.float64)
        self.store[(field, level)] = a.reshape(3, -1) if field in VECTOR_FIELDS else a.ravel()

    def get(self, field, level):
        return self.store[(field, level)]


@pytest.mark.parametrize("nranks", [1, 2, 3, 5])
def test_slab_group_set_and_get_round_trip_whole_arrays(nranks):
    from hpcrack_b200.slab import SlabGroup, local_part
    from hpcrack_b200.solver import U, D

    ml, enb = 2, (2, 3, 4)
    g = object.__new__(SlabGroup)
    g.maxlevel, g.enb, g.nranks = ml, enb, nranks
    g.dims = [tuple(e * (1 << l) + 1 for e in enb) for l in range(ml + 1)]
    g.ranks = [_FakeRank(ml, enb, nranks, r) for r in range(nranks)]
    g.run = lambda fn: [fn(h) for h in g.ranks]
    rng = np.random.default_rng(2)
    for l in range(ml + 1):
        n = int(np.prod(g.dims[l]))
        d, u = rng.standard_normal(n), rng.standard_normal((3, n))
        g.set(D, l, d)
        g.set(U, l, u)
        assert np.array_equal(g.get(D, l), d)
        assert np.array_equal(g.get(U, l), u)
        for h in g.ranks:  # every rank holds its planes, ghost planes included
            nz, zb, _, _ = h.plans[l]
            nx, ny = g.dims[l][:2]
            assert np.array_equal(h.get(D, l), d.reshape(-1, ny, nx)[zb:zb + nz].ravel())
            assert np.array_equal(h.get(D, l), local_part(h, l, d))
            assert np.array_equal(h.get(U, l), local_part(h, l, u, vector=True))


def test_slab_group_run_aborts_and_reraises_the_failing_rank():
    """SlabGroup.run: every rank's call runs in its own thread; a rank that raises aborts the group
    (no device here: aborting a null group is a refused call, not a crash) and its own exception is
    re-raised, not the errors of ranks whose waits the abort ended."""
    from hpcrack_b200.slab import SlabGroup

    g = object.__new__(SlabGroup)
    g.lib = L.load()
    g.group = None
    g.ranks = [_FakeRank(1, (2, 2, 4), 3, r) for r in range(3)]

    def fn(h):
        r = h.slab[1]
        if r == 1:
            raise ValueError("rank 1 failed")
        if r == 2:
            raise RuntimeError("slab group aborted by another rank")
        return r

    with pytest.raises(ValueError, match="rank 1 failed"):
        g.run(fn)
    assert g.run(lambda h: h.slab[1] * 10) == [0, 10, 20]


def test_slab_footprints_let_a_specimen_exceed_one_gpu():
    """hpc_footprint_slab: a rank holds its planes (plus the gathered coarsest level), so the split's
    per-rank bytes shrink with the rank count.  1025^3 (every form's buffers: ~920 GB) fits 8 GPUs of
    180 GB; 2049^3 (8.6e9 nodes) is past the 2^31-node limit of one context, refused whole and
    accepted split over 64 ranks, each under 180 GB."""
    from hpcrack_b200.solver import Hierarchy

    whole = Hierarchy.footprint(5, (8, 8, 8))
    assert Hierarchy.footprint(5, (8, 8, 8), slab=(1, 0)) == whole
    for n in (2, 4, 8):
        parts = [Hierarchy.footprint(5, (8, 8, 8), slab=(n, r)) for r in range(n)]
        assert max(parts) < whole * (1.0 / n + 0.08), (n, max(parts), whole)
        assert sum(parts) >= whole
    big = Hierarchy.footprint(7, (8, 8, 8))
    assert big > 180e9
    assert all(Hierarchy.footprint(7, (8, 8, 8), slab=(8, r)) < 180e9 for r in range(8))
    with pytest.raises(L.HpcError):  # 2049^3 as 64^3 coarsest elements: 64 ranks own a coarsest plane each
        Hierarchy.footprint(5, (64, 64, 64))
    assert all(Hierarchy.footprint(5, (64, 64, 64), slab=(64, r)) < 180e9 for r in (0, 1, 63))
    with pytest.raises(L.HpcError):  # 9 coarsest planes cannot go to 10 ranks (initialization.cpp:50-72)
        Hierarchy.footprint(5, (8, 8, 8), slab=(10, 0))


def test_slab_group_lifecycle_without_a_device():
    """The in-process group is host state: create, refuse bad joins, abort, destroy - no device needed."""
    import ctypes as C

    lib = L.load()
    g = C.c_void_p()
    assert lib.hpc_slab_group_create(C.byref(g), 0) == 1          # HPC_ERR_ARG: no ranks
    assert lib.hpc_slab_group_create(C.byref(g), 65) == 1         # beyond the group's rank table
    assert lib.hpc_slab_group_create(C.byref(g), 3) == 0
    assert lib.hpc_slab_group_join(g, None) == 1                  # no context
    assert lib.hpc_slab_group_join(None, None) == 1
    assert lib.hpc_slab_group_abort(g) == 0
    assert lib.hpc_slab_group_abort(None) == 1
    assert lib.hpc_slab_group_destroy(g) == 0
    assert lib.hpc_slab_group_destroy(None) == 0
    assert lib.hpc_slab_join_nccl(None, None) == 1
    out = (C.c_int * 4)()
    assert lib.hpc_slab_level(None, 2, 0, 0, out) == 1
