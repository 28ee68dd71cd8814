"""A slab FAS V-cycle over gloo ranks (world sizes 2 and 3) against the same cycle on the whole grid (CPU).

The cycle follows the library's z split step by step, with numpy standing in for the kernels and a
7-point operator for the element operator:

- every level's planes, ghost planes and owned planes come from hpc_slab_level (the library's plan);
- coarse plane kc lies on fine plane 2 kc + zsh (zsh = 2 zb_coarse - zb_fine);
- ghost planes are exchanged where the library exchanges them (slab.cu, after the reference's SendRecv
  sites): the PCG direction after every update, the coarse u and u_old after injection, the fine
  residual before the FAS restriction, the fine u after prolongation;
- dot products sum owned planes and are all-reduced;
- the coarsest level is gathered from every rank and solved redundantly (the one-block solver's part).

FAS as cycle_u does it (mechanical_multigrid.cpp:18-54): pre-smoothing by restarted Jacobi-PCG,
u_c = u_f(2i) (solution_injection), f_c = A_c u_c + full weighting of r_f (coarsen_f_standard_routine,
weights 1, 1/2, 1/4, 1/8), the coarse cycle, u_f += P(u_c - u_c_old) (refine_standard_routine),
post-smoothing.  Two cycles on 2 and 3 ranks reproduce the whole-grid cycles to 1e-12.
"""
import os
import socket

import numpy as np
import pytest

from hpcrack_b200.solver import slab_level

torch = pytest.importorskip("torch")

ML, ENB = 2, (2, 2, 4)  # levels 3x3x5, 5x5x9, 9x9x17 nodes
NU0, NU1, NU2, CYCLES = 12, 3, 3, 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _apply(u, scale=1.0):
    """scale (6u - the sum of the 6 neighbours), zero outside the array.  Level l of a hierarchy with
    finest level L takes scale 2^(L - l): the Galerkin coarse operator of this stencil under the
    restriction weights 1, 1/2, 1/4, 1/8 (a Q1 stiffness grows with the spacing in 3-D)."""
    out = 6.0 * u
    for ax in range(3):
        hi = [slice(None)] * 3
        lo = [slice(None)] * 3
        hi[ax], lo[ax] = slice(1, None), slice(None, -1)
        out[tuple(hi)] -= u[tuple(lo)]
        out[tuple(lo)] -= u[tuple(hi)]
    return scale * out


def _scale(l):
    return float(2 ** (ML - l))


class Comm:
    """One rank's plans and exchanges; the whole grid is the one-rank case (no exchange)."""

    def __init__(self, nranks, rank, dist=None):
        self.nranks, self.rank, self.dist = nranks, rank, dist
        self.plan = [slab_level(ML, ENB, nranks, rank, l) for l in range(ML + 1)]

    def dot(self, l, a, b):
        _, _, lo, hi = self.plan[l]
        s = float(np.sum(a[lo:hi] * b[lo:hi]))
        if self.nranks == 1:
            return s
        t = torch.tensor([s], dtype=torch.float64)
        self.dist.all_reduce(t)
        return float(t[0])

    def halo(self, l, v):
        if self.nranks == 1:
            return
        d, r, nz = self.dist, self.rank, self.plan[l][0]
        reqs, bufs = [], []
        if r > 0:
            reqs.append(d.isend(torch.from_numpy(np.ascontiguousarray(v[1])), r - 1))
            bufs.append((0, torch.empty(v[0].shape, dtype=torch.float64)))
            reqs.append(d.irecv(bufs[-1][1], r - 1))
        if r < self.nranks - 1:
            reqs.append(d.isend(torch.from_numpy(np.ascontiguousarray(v[nz - 2])), r + 1))
            bufs.append((nz - 1, torch.empty(v[0].shape, dtype=torch.float64)))
            reqs.append(d.irecv(bufs[-1][1], r + 1))
        for q in reqs:
            q.wait()
        for k, b in bufs:
            v[k] = b.numpy()

    def gather(self, l, v):
        """The whole level from every rank's owned planes."""
        nz, zb, lo, hi = self.plan[l]
        if self.nranks == 1:
            return v.copy()
        parts = [None] * self.nranks
        self.dist.all_gather_object(parts, (zb + lo, v[lo:hi].copy()))
        return np.concatenate([p for _, p in sorted(parts, key=lambda t: t[0])], axis=0)


def _pcg(comm, l, u, f, nb):
    """Restarted Jacobi-PCG (mechanical_pcg.cpp:268-321): r = f - A u, then nb iterations."""
    r = f - _apply(u, _scale(l))
    p = np.zeros_like(u)
    rz_old = None
    for i in range(nb):
        z = r / (6.0 * _scale(l))
        rz = comm.dot(l, r, z)
        p = z if i == 0 else z + (rz / rz_old) * p
        comm.halo(l, p)
        w = _apply(p, _scale(l))
        alpha = rz / comm.dot(l, p, w)
        u += alpha * p
        r -= alpha * w
        rz_old = rz
    return r


def _zsh(comm, l):
    return 2 * comm.plan[l - 1][1] - comm.plan[l][1]


def _restrict(rf, nzc, zsh):
    """Full weighting at fine plane 2 kc + zsh (x, y at 2i, 2j), zero outside the array."""
    nzf, ny, nx = rf.shape
    p = np.zeros((nzf + 2, ny + 2, nx + 2))
    p[1:-1, 1:-1, 1:-1] = rf
    out = np.zeros((nzc, (ny + 1) // 2, (nx + 1) // 2))
    for kc in range(nzc):
        fz = 2 * kc + zsh
        if fz < 0:
            continue  # a ghost plane: the exchange fills it
        acc = 0.0
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    w = 0.5 ** (abs(dz) + abs(dy) + abs(dx))
                    acc = acc + w * p[fz + 1 + dz, 1 + dy:ny + 1 + dy:2, 1 + dx:nx + 1 + dx:2]
        out[kc] = acc
    return out


def _prolong_axis(c, n_fine, shift, axis):
    """Linear interpolation along one axis: fine i from coarse (i - shift) / 2, on global parity."""
    c = np.moveaxis(c, axis, 0)
    out = np.empty((n_fine,) + c.shape[1:])
    for i in range(n_fine):
        q = i - shift
        kc = (q + 1) >> 1
        out[i] = c[kc] if q % 2 == 0 else 0.5 * (c[kc] + c[kc - 1])
    return np.moveaxis(out, 0, axis)


def _cycle(comm, l, u, f):
    if l == 0:
        uw, fw = comm.gather(0, u), comm.gather(0, f)
        _pcg(Comm(1, 0), 0, uw, fw, NU0)  # the same whole level, the same solution on every rank
        nz, zb, _, _ = comm.plan[0]
        u[:] = uw[zb:zb + nz]
        return
    r = _pcg(comm, l, u, f, NU1)
    zsh = _zsh(comm, l)
    nzc = comm.plan[l - 1][0]
    uc = np.zeros((nzc,) + tuple((s + 1) // 2 for s in u.shape[1:]))
    for kc in range(nzc):
        if 2 * kc + zsh >= 0:
            uc[kc] = u[2 * kc + zsh, ::2, ::2]
    comm.halo(l - 1, uc)
    ucold = uc.copy()
    comm.halo(l, r)
    fc = _apply(uc, _scale(l - 1)) + _restrict(r, nzc, zsh)
    _cycle(comm, l - 1, uc, fc)
    e = uc - ucold
    e = _prolong_axis(e, u.shape[0], zsh, 0)
    e = _prolong_axis(e, u.shape[1], 0, 1)
    e = _prolong_axis(e, u.shape[2], 0, 2)
    u += e
    comm.halo(l, u)
    _pcg(comm, l, u, f, NU2)


def _global_f():
    dims = [((ENB[2] << ML) + 1), ((ENB[1] << ML) + 1), ((ENB[0] << ML) + 1)]
    return np.random.default_rng(9).standard_normal(dims)


def _solve(comm, f):
    u = np.zeros_like(f)
    for _ in range(CYCLES):
        _cycle(comm, ML, u, f)
    return u


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        comm = Comm(world, rank, dist)
        nz, zb, lo, hi = comm.plan[ML]
        f = _global_f()[zb:zb + nz].copy()
        u = _solve(comm, f)
        q.put((rank, zb + lo, u[lo:hi].copy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_fas_vcycles_over_gloo_reproduce_the_whole_grid(world):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    whole = _solve(Comm(1, 0), _global_f())
    split = np.concatenate([u for _, _, u in res], axis=0)
    assert [z0 for _, z0, _ in res][0] == 0 and split.shape == whole.shape
    # the cycles did work: the residual fell by orders of magnitude
    f = _global_f()
    assert np.linalg.norm(f - _apply(whole, _scale(ML))) < 1e-2 * np.linalg.norm(f)
    err = np.linalg.norm(split - whole) / np.linalg.norm(whole)
    assert err < 1e-12, err
