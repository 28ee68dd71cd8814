"""Restartable history dumps in the reference's file format.

The reference dumps the finest u, v, w, H and d every ``Tdatafrequence`` increments
(crack_propagation.cpp:99-106) with ``write_vector_3D`` (write_read_history.cpp:18-53): one file
``Time_step_data/<name>_t_<t>_Proc_<rank>.dat`` per field holding the grid's nx*ny*nz doubles,
x fastest, in the machine's byte order, no header; ``read_vector_3D`` (:55-86) reads the same.
Those five files alone do not restart the loop - the load state (Ut, dU, u_proportion, Ue, f_norm,
fd_norm) and d_old are missing - so two more files of the same kind sit beside them:
``dold_t_<t>_Proc_<rank>.dat`` (d_old, nx*ny*nz doubles) and ``state_t_<t>_Proc_<rank>.dat`` (the
six loop scalars in :func:`Hierarchy.state` order).
"""
from __future__ import annotations

import os

import numpy as np

FIELD_FILES = (("u", "u"), ("v", "v"), ("w", "w"), ("H", "H"), ("d", "d"), ("d_old", "dold"))


def dump_path(directory: str, name: str, t: int, rank: int = 0) -> str:
    """write_read_history.cpp:27: ``Time_step_data/%s_t_%d_Proc_%d.dat``."""
    return os.path.join(directory, "Time_step_data", f"{name}_t_{t}_Proc_{rank}.dat")


def write_vector_3d(path: str, arr: np.ndarray) -> None:
    np.ascontiguousarray(arr, dtype=np.float64).tofile(path)


def read_vector_3d(path: str, n: int) -> np.ndarray:
    a = np.fromfile(path, dtype=np.float64)
    if a.size != n:
        raise ValueError(f"{path}: {a.size} doubles, expected {n}")
    return a


def write_checkpoint(directory: str, t: int, fields: dict, state6, rank: int = 0) -> list:
    """Writes the five reference dumps plus d_old and the loop state; returns the paths."""
    os.makedirs(os.path.join(directory, "Time_step_data"), exist_ok=True)
    paths = []
    for key, name in FIELD_FILES:
        p = dump_path(directory, name, t, rank)
        write_vector_3d(p, fields[key])
        paths.append(p)
    p = dump_path(directory, "state", t, rank)
    write_vector_3d(p, np.asarray(state6, dtype=np.float64).reshape(6))
    paths.append(p)
    return paths


def read_checkpoint(directory: str, t: int, n: int, rank: int = 0):
    """-> ({u, v, w, H, d, d_old}, state6) as written by :func:`write_checkpoint`."""
    fields = {key: read_vector_3d(dump_path(directory, name, t, rank), n) for key, name in FIELD_FILES}
    state = read_vector_3d(dump_path(directory, "state", t, rank), 6)
    return fields, list(state)
