"""One specimen split along z over ranks (the reference's MPI domain decomposition, in z).

Each rank is a slab context (``Hierarchy(..., slab=(nranks, rank))``, hpc_create_slab) holding its
planes of every level plus one ghost plane towards each neighbour (initialization.cpp:19-134).  The
library exchanges ghost planes at the reference's SendRecv sites (mpi_communications.h:24-47) and
combines every reduction over the ranks (pcg_utilities.cpp:16-58).  Two transports:

- :class:`SlabGroup` - all ranks in this process, one host thread each (one GPU or several): the
  in-process transport of the library.  It also stands behind the :class:`Hierarchy` interface, so a
  split specimen is driven like a whole one (``set``/``get`` take and return whole-specimen arrays).
- :func:`join_nccl` / :func:`from_process_group` - one process per GPU over NCCL.
"""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import lib as _L
from .solver import VECTOR_FIELDS, Hierarchy, slab_level

__all__ = ["SlabGroup", "slab_level", "local_part", "nccl_unique_id", "join_nccl", "from_process_group"]


def _planes(arr, nz_total, ny, nx, vector):
    a = np.asarray(arr, dtype=np.float64)
    return a.reshape((3, nz_total, ny, nx) if vector else (nz_total, ny, nx))


class SlabGroup:
    """A specimen split along z over `nranks` slab contexts of this process.

    Calls other than ``set``/``get`` run on every rank at once (one thread per rank: each one is a
    collective step) and return rank 0's result; :meth:`step` also checks that every rank returned the
    same outputs.  ``devices``: device of each rank, cycled (default: all on device 0)."""

    def __init__(self, maxlevel, enb, nranks, x0=(0.0, 0.0, 0.0), roi=(0, 0, 0), devices=(0,)):
        self.lib = _L.load()
        self.maxlevel = int(maxlevel)
        self.enb = tuple(int(e) for e in enb)
        self.nranks = int(nranks)
        self.dims = [tuple(e * (1 << l) + 1 for e in self.enb) for l in range(self.maxlevel + 1)]
        g = C.c_void_p()
        _L.check("hpc_slab_group_create", self.lib.hpc_slab_group_create(C.byref(g), self.nranks))
        self.group = g
        self.ranks: list[Hierarchy] = []
        try:
            for r in range(self.nranks):
                h = Hierarchy(self.maxlevel, self.enb, x0, roi, device=int(devices[r % len(devices)]),
                              slab=(self.nranks, r))
                self.ranks.append(h)
                _L.check("hpc_slab_group_join", self.lib.hpc_slab_group_join(self.group, h.h))
        except BaseException:
            self.close()
            raise

    # ------------------------------------------------------------ lifetime
    def close(self):
        for h in getattr(self, "ranks", []):
            h.close()
        self.ranks = []
        if getattr(self, "group", None):
            self.lib.hpc_slab_group_destroy(self.group)
            self.group = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ collective calls
    def run(self, fn):
        """fn(rank_hierarchy) on every rank at once; the results in rank order.  A rank that raises
        aborts the group (the others' waits end) and its exception is re-raised."""
        n = len(self.ranks)
        out = [None] * n
        err: list = [None] * n

        def work(r):
            try:
                out[r] = fn(self.ranks[r])
            except BaseException as e:  # noqa: BLE001 - handed to the caller below
                err[r] = e
                self.lib.hpc_slab_group_abort(self.group)

        ts = [threading.Thread(target=work, args=(r,)) for r in range(n)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        first = [e for e in err if e is not None]
        if first:
            # the rank that failed first, not a rank whose wait the abort ended
            own = [e for e in first if "aborted" not in str(e)]
            raise (own or first)[0]
        return out

    def __getattr__(self, name):
        attr = getattr(Hierarchy, name, None)
        if name.startswith("_") or not callable(attr):
            raise AttributeError(name)

        def call(*a, **k):
            return self.run(lambda h: getattr(h, name)(*a, **k))[0]

        return call

    def step(self, *a, **k):
        outs = self.run(lambda h: h.step(*a, **k))
        for o in outs[1:]:
            if o != outs[0]:
                raise RuntimeError(f"slab ranks disagree on the step outputs: {outs}")
        return outs[0]

    # ------------------------------------------------------------ whole-specimen fields
    def n(self, level):
        d = self.dims[level]
        return d[0] * d[1] * d[2]

    def set(self, field, level, arr):
        nx, ny, nz = self.dims[level]
        vec = field in VECTOR_FIELDS
        a = _planes(arr, nz, ny, nx, vec)

        def put(h):
            lnz, zb, _, _ = h.plans[level]
            part = a[:, zb:zb + lnz] if vec else a[zb:zb + lnz]
            h.set(field, level, np.ascontiguousarray(part))

        self.run(put)

    def get(self, field, level):
        nx, ny, nz = self.dims[level]
        vec = field in VECTOR_FIELDS
        out = np.empty((3, nz, ny, nx) if vec else (nz, ny, nx))
        for h in self.ranks:
            lnz, zb, lo, hi = h.plans[level]
            loc = h.get(field, level).reshape((3, lnz, ny, nx) if vec else (lnz, ny, nx))
            if vec:
                out[:, zb + lo:zb + hi] = loc[:, lo:hi]
            else:
                out[zb + lo:zb + hi] = loc[lo:hi]
        return out.reshape(3, -1) if vec else out.ravel()

    def set_choice(self, level, arr):
        nx, ny, nz = self.dims[level]
        a = np.asarray(arr, dtype=np.int16).reshape(nz, ny, nx)
        def put(h):
            lnz, zb, _, _ = h.plans[level]
            h.set_choice(level, np.ascontiguousarray(a[zb:zb + lnz]))

        self.run(put)

    def get_choice(self, level):
        nx, ny, nz = self.dims[level]
        out = np.empty((nz, ny, nx), dtype=np.int16)
        for h in self.ranks:
            lnz, zb, lo, hi = h.plans[level]
            out[zb + lo:zb + hi] = h.get_choice(level).reshape(lnz, ny, nx)[lo:hi]
        return out.ravel()


# ---------------------------------------------------------------- one process per GPU
def local_part(h: Hierarchy, level, arr, vector=False):
    """A slab rank's planes (ghost planes included) of a whole-specimen array of `level`."""
    nx, ny, _ = h.dims[level]
    nz, zb, _, _ = h.plans[level]
    a = np.asarray(arr)
    a = a.reshape((3, -1, ny, nx) if vector else (-1, ny, nx))
    return np.ascontiguousarray(a[:, zb:zb + nz] if vector else a[zb:zb + nz]).reshape((3, -1) if vector else -1)


def nccl_unique_id() -> bytes:
    """hpc_nccl_unique_id: the id rank 0 makes and hands to every rank."""
    lib = _L.load()
    buf = (C.c_ubyte * 128)()
    _L.check("hpc_nccl_unique_id", lib.hpc_nccl_unique_id(buf))
    return bytes(buf)


def join_nccl(h: Hierarchy, uid: bytes):
    """hpc_slab_join_nccl: the slab context of this process joins the NCCL communicator (every rank at
    once)."""
    if h.slab is None:
        raise ValueError("join_nccl needs a slab context")
    buf = (C.c_ubyte * 128).from_buffer_copy(uid)
    _L.check("hpc_slab_join_nccl", h.lib.hpc_slab_join_nccl(h.h, buf))


def from_process_group(maxlevel, enb, x0=(0.0, 0.0, 0.0), roi=(0, 0, 0), device=None) -> Hierarchy:
    """This process's slab of a specimen split over the ranks of torch.distributed's default group
    (initialised by the caller): rank 0's NCCL id reaches the others through the group."""
    import torch.distributed as dist

    rank, world = dist.get_rank(), dist.get_world_size()
    h = Hierarchy(maxlevel, enb, x0, roi, device=rank if device is None else device, slab=(world, rank))
    box = [nccl_unique_id() if rank == 0 else None]
    dist.broadcast_object_list(box, src=0)
    join_nccl(h, box[0])
    return h
