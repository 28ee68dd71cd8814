"""Scenario builders shared by the parity tests: the same seeded inputs are loaded into any
implementation exposing the common field API (the CUDA library's Hierarchy, the C oracle
COracle, the compiled reference RefOracle)."""
from __future__ import annotations

import numpy as np

from hpcrack_b200 import microstructure as ms

BULK, G, GC, D, H, FD, KE, GE, R, DOLD, DOLDF = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10
U, FU, RU, UOLD = 16, 17, 18, 19


def rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def random_level_fields(rng, n, zero_frac=0.15):
    """Random positive moduli, a phase field in [-0.1, 1.1] with exact zeros (the zero rule of
    gauss_point_MP), history, element moduli, regimes and displacements for one level of n nodes."""
    f = {
        BULK: rng.uniform(1.0, 2.0, n),
        G: rng.uniform(0.5, 1.0, n),
        GC: rng.uniform(0.1, 0.3, n),
        D: np.where(rng.random(n) < zero_frac, 0.0, rng.uniform(-0.1, 1.1, n)),
        H: rng.uniform(0.0, 1.0, n),
        KE: rng.uniform(1.0, 2.0, n),
        GE: rng.uniform(0.5, 1.0, n),
    }
    return f


def load_random(impls, maxlevel, enb, seed, with_zero_material=False):
    """Loads identical random fields into every implementation; returns the arrays."""
    rng = np.random.default_rng(seed)
    data = []
    dims = [tuple(e * (1 << l) + 1 for e in enb) for l in range(maxlevel + 1)]
    for l in range(maxlevel + 1):
        n = int(np.prod(dims[l]))
        f = random_level_fields(rng, n)
        if with_zero_material:
            f[BULK][rng.random(n) < 0.01] = 0.0
        ch = rng.integers(0, 3, n).astype(np.int16)
        u = rng.standard_normal((3, n))
        fu = rng.standard_normal((3, n))
        for impl in impls:
            for k, v in f.items():
                impl.set(k, l, v)
            impl.set_choice(l, ch)
            impl.set(U, l, u)
            impl.set(FU, l, fu)
        data.append((f, ch, u, fu))
    return data


def load_workload(impls, w: ms.Workload):
    """Image material + pre-crack of a workload into every implementation (the oracle's image
    path for oracles, the GPU input kernel for the library)."""
    nx, ny, nz = w.nodes
    Hc, dc = ms.precrack_fields(w)
    for impl in impls:
        impl.image_material(w.image, (nx, ny, nz), w.table(), w.voxel_size)
        if w.crack:
            impl.set(H, w.maxlevel, Hc)
            impl.set(D, w.maxlevel, dc)
            impl.voigt_all_level(H)
