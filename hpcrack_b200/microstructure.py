"""Synthetic inclusion microstructures and their material tables (host logic).

The reference reads a raw uint8 voxel image, x fastest (image_input.cpp:33-76),
and maps gray levels to (E, nu, Gc) through data/Material_Property.csv
(csv_reader.cpp:14-63, image_input.cpp:120-142).  No public dataset is named
for this path, so seeded synthetic images stand in: non-overlapping spheres
placed by rejection sampling in a matrix.  Labels map to gray levels
0 (matrix), 85 (pore) and 170 (inclusion); the material table uses the
breakpoint pairs 0,84 | 85,169 | 170,255 so that the reference's
integer-division gray-level interpolation (image_input.cpp:134-137) lands
exactly on each phase's row.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

MATRIX_GRAY, PORE_GRAY, INCLUSION_GRAY = 0, 85, 170
GRAY_BREAKPOINTS = (0, 84, 85, 169, 170, 255)


@dataclasses.dataclass
class Phase:
    """A population of spheres of one label."""
    gray: int
    rmin: float
    rmax: float
    count: int | None = None          # fixed number of spheres, or
    volume_fraction: float | None = None  # target volume fraction of the box


@dataclasses.dataclass
class Material:
    E: float    # Pa
    nu: float
    gc: float   # N/m


MATRIX = Material(30e9, 0.2, 50.0)
INCLUSION = Material(70e9, 0.25, 100.0)
PORE = Material(1e9, 0.2, 50.0)  # pore nu and Gc are unspecified: matrix values


def material_table(matrix: Material = MATRIX, pore: Material = PORE, inclusion: Material = INCLUSION):
    """(gray, E, nu, gc) columns in the CSV layout of data/Material_Property.csv."""
    gray = list(GRAY_BREAKPOINTS)
    mats = [matrix, matrix, pore, pore, inclusion, inclusion]
    return (gray, [m.E for m in mats], [m.nu for m in mats], [m.gc for m in mats])


def write_material_csv(path: str, table) -> None:
    gray, E, nu, gc = table
    with open(path, "w") as f:
        f.write("Gray level," + ",".join(str(int(g)) for g in gray) + "\n")
        f.write("E/Pa," + ",".join(repr(float(v)) for v in E) + "\n")
        f.write("nu," + ",".join(repr(float(v)) for v in nu) + "\n")
        f.write("gc/(N/m)," + ",".join(repr(float(v)) for v in gc) + "\n")


def sphere_image(shape, seed: int, phases, matrix_gray: int = MATRIX_GRAY, max_tries: int = 200000) -> np.ndarray:
    """uint8 image of shape (nz, ny, nx) (x fastest when flattened) with non-overlapping spheres.

    Centres are uniform in the box, radii uniform in [rmin, rmax]; a candidate is rejected if it
    overlaps any sphere already placed (of any phase).  Phases are placed in order until their
    count or volume fraction is reached.
    """
    nx, ny, nz = (int(s) for s in shape)
    rng = np.random.default_rng(seed)
    img = np.full((nz, ny, nx), matrix_gray, dtype=np.uint8)
    centres = np.zeros((0, 3))
    radii = np.zeros(0)
    box = float(nx) * ny * nz
    for ph in phases:
        placed_vol = 0.0
        placed = 0
        tries = 0
        while tries < max_tries:
            if ph.count is not None and placed >= ph.count:
                break
            if ph.volume_fraction is not None and placed_vol >= ph.volume_fraction * box:
                break
            tries += 1
            r = rng.uniform(ph.rmin, ph.rmax)
            c = rng.uniform((0.0, 0.0, 0.0), (nx - 1, ny - 1, nz - 1))
            if len(radii):
                d2 = np.sum((centres - c) ** 2, axis=1)
                if np.any(d2 < (radii + r) ** 2):
                    continue
            centres = np.vstack([centres, c])
            radii = np.append(radii, r)
            _paint(img, c, r, ph.gray)
            placed += 1
            placed_vol += 4.0 / 3.0 * math.pi * r ** 3
    return img


def _paint(img, c, r, gray):
    nz, ny, nx = img.shape
    lo = [max(0, int(math.floor(c[a] - r))) for a in range(3)]
    hi = [min(n, int(math.ceil(c[a] + r)) + 1) for a, n in zip(range(3), (nx, ny, nz))]
    if any(h <= l for l, h in zip(lo, hi)):
        return
    z, y, x = np.meshgrid(np.arange(lo[2], hi[2]), np.arange(lo[1], hi[1]), np.arange(lo[0], hi[0]), indexing="ij")
    m = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 < r * r
    sub = img[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
    sub[m] = gray


def maxlevel_for(voxel_nx: int, roi_x: int, element_nb_x: int) -> int:
    """main.cpp:52-68: levels from the X axis only."""
    nb_f = voxel_nx - roi_x - 1
    nb_c = element_nb_x
    if 2 * nb_c > nb_f:
        return 0
    lvl = 0
    while True:
        nb_c *= 2
        if nb_c <= nb_f:
            lvl += 1
        else:
            break
    return lvl


@dataclasses.dataclass
class Workload:
    """One specimen: image, geometry and the staggered-loop parameters."""
    name: str
    image: np.ndarray            # (nz, ny, nx) uint8
    element_nb: tuple
    maxlevel: int
    x_start: tuple
    voxel_size: float
    lc: float                    # length scale l in finest-element units times h (main.cpp:94)
    small_k: float
    mg_u: tuple                  # (nu0, nu1, nu2, gamma, ncy)
    mg_d: tuple
    increments: int
    ut0: float = 0.0             # <= 0: the reference's Ue-based schedule
    du: float = 0.0
    du_factor: float = 1.5e-3
    mech_tol: float = 1e-6       # squared ratio |r|^2/|f|^2
    pf_tol: float = 1e-12
    crack: dict | None = None    # pre-crack description (H, d planes)

    @property
    def nodes(self):
        nz, ny, nx = self.image.shape
        return (nx, ny, nz)

    def table(self):
        return material_table()


def hierarchy_for(nodes) -> tuple:
    """(maxlevel, element_nb) for a box of `nodes` per axis: the deepest hierarchy whose coarsest
    level keeps at least 8 elements on the shortest axis (a 9-node coarsest grid, as the
    reference's configurations use) with every axis divisible by 2^maxlevel."""
    elems = [int(n) - 1 for n in nodes]
    L = 0
    while all(e % (1 << (L + 1)) == 0 for e in elems) and min(elems) >> (L + 1) >= 8:
        L += 1
    return L, tuple(e >> L for e in elems)


def inclusion_workload(name: str, nodes, seed: int, volume_fraction: float, maxlevel: int | None,
                       increments: int) -> Workload:
    """A two-phase inclusion specimen of the batched / served mixes: spheres with radii in [4, 8]
    voxels scaled by the shortest axis / 64, to `volume_fraction`; materials, length scale and
    load schedule of the 65^3 configuration; tolerance |r|/|f| <= 1e-8 (squared 1e-16)."""
    nx, ny, nz = (int(n) for n in nodes)
    s = (min(nx, ny, nz) - 1) / 64.0
    img = sphere_image((nx, ny, nz), seed, [Phase(INCLUSION_GRAY, max(4 * s, 1.5), max(8 * s, 2.0),
                                                  volume_fraction=volume_fraction)])
    if maxlevel is None:
        maxlevel, enb = hierarchy_for((nx, ny, nz))
    else:
        enb = tuple((n - 1) >> maxlevel for n in (nx, ny, nz))
    return Workload(name, img, enb, maxlevel, (0.0, 0.0, 0.0), 1e-6, 2.0, 1e-6, (50, 4, 2, 1, 200),
                    (10, 2, 1, 1, 200), increments, ut0=1e-4 * (nz - 1), du=1e-4 * (nz - 1), mech_tol=1e-16,
                    pf_tol=1e-16)


def make_workload(name: str) -> Workload:
    """Seeded synthetic stand-ins for the benchmark configurations.

    * ``parity65``  65^3, seed 0, 12 spheres r in [4,8]; element_nb 8 (levels 9/17/33/65);
      3 increments of 1e-4*Nz top displacement; tolerance |r|/|f| <= 1e-8.
    * ``plain257``  257^3, seed 1, inclusions r in [6,20] to 25 %, pores r in [3,8] to 5 %;
      pre-crack at mid-height over half the x width; 20 increments.
    * ``mid129`` / ``mid193``  the plain257 recipe scaled to 129^3 / 193^3 (193: element_nb 12), for
      profiling at a few GB of device memory.
    * ``crack33`` / ``crack65``  the plain257 recipe (three phases, pre-crack) scaled to 33^3 / 65^3,
      the parity cases of the benchmarked configuration (the reference finishes them in minutes).
    * ``large513``  513^3, seed 2, inclusions to 30 %.
    * ``small17`` / ``small33`` test-sized variants of parity65; ``parity129`` the same recipe at 129^3
      (the CPU baseline's second full-run size).
    """
    if name in ("parity65", "parity129", "small17", "small33"):
        n = {"parity65": 65, "parity129": 129, "small17": 17, "small33": 33}[name]
        scale = (n - 1) / 64.0
        img = sphere_image((n, n, n), 0, [Phase(INCLUSION_GRAY, 4 * scale, 8 * scale, count=12)])
        return Workload(name, img, (8, 8, 8), maxlevel_for(n, 0, 8), (0.0, 0.0, 0.0), 1e-6, 2.0, 1e-6,
                        (50, 4, 2, 1, 200), (10, 2, 1, 1, 200), 3, ut0=1e-4 * (n - 1), du=1e-4 * (n - 1),
                        mech_tol=1e-16, pf_tol=1e-16)
    if name in ("plain257", "mid129", "mid193", "crack33", "crack65"):
        n = {"plain257": 257, "mid129": 129, "mid193": 193, "crack33": 33, "crack65": 65}[name]
        enb = 12 if n == 193 else 8  # 193 = 12 * 2^4 + 1
        s = (n - 1) / 256.0
        # radii floors only bind below 129^3 (crack33 / crack65 keep spheres a few voxels wide)
        img = sphere_image((n, n, n), 1, [Phase(INCLUSION_GRAY, max(6 * s, 2.0), max(20 * s, 4.0),
                                                volume_fraction=0.25),
                                          Phase(PORE_GRAY, max(3 * s, 1.5), max(8 * s, 2.5), volume_fraction=0.05)])
        return Workload(name, img, (enb, enb, enb), maxlevel_for(n, 0, enb), (0.0, 0.0, 0.0), 1e-6, 2.0, 1e-6,
                        (50, 4, 2, 1, 200), (10, 2, 1, 1, 200), 20, ut0=1e-4 * (n - 1), du=1e-4 * (n - 1),
                        mech_tol=1e-16, pf_tol=1e-16, crack={"H": 1e6, "layer": (n - 1) // 2, "xfrac": 0.5})
    if name == "large513":
        n = 513
        img = sphere_image((n, n, n), 2, [Phase(INCLUSION_GRAY, 6, 20, volume_fraction=0.30)])
        return Workload(name, img, (8, 8, 8), maxlevel_for(n, 0, 8), (0.0, 0.0, 0.0), 1e-6, 2.0, 1e-6,
                        (50, 4, 2, 1, 200), (10, 2, 1, 1, 200), 5, ut0=1e-4 * (n - 1), du=1e-4 * (n - 1),
                        mech_tol=1e-16, pf_tol=1e-16)
    raise KeyError(name)


def precrack_fields(w: Workload):
    """Initial H (element field) and d (nodal) of a planar pre-crack: element layer `layer`, elements
    with x index below xfrac*(nx-1), all y; H = H_crack there (as initial_crack, strain_history.cpp:30-70,
    does for its planes) and d = 1 on the nodes of those elements."""
    nx, ny, nz = w.nodes
    H = np.zeros((nz, ny, nx))
    d = np.zeros((nz, ny, nx))
    if not w.crack:
        return H.ravel(), d.ravel()
    k = int(w.crack["layer"])
    xe = int(w.crack["xfrac"] * (nx - 1))
    H[k, : ny - 1, :xe] = float(w.crack["H"])
    d[k : k + 2, :, : xe + 1] = 1.0
    return H.ravel(), d.ravel()


def write_inputs(w: Workload, directory: str, extra: dict | None = None) -> dict:
    """Writes the reference's inputs for this workload: raw image, data/Material_Property.csv and a
    config.txt (keys written without spaces around '=', which the reference's parser requires;
    configuration.cpp:25 compares the whole text left of '=').  `extra` adds key=value lines
    (e.g. outTdata, Tdatafrequence, outK)."""
    os.makedirs(os.path.join(directory, "data"), exist_ok=True)
    raw = os.path.join(directory, "data", f"{w.name}.raw")
    w.image.tofile(raw)
    write_material_csv(os.path.join(directory, "data", "Material_Property.csv"), w.table())
    nx, ny, nz = w.nodes
    cfg = os.path.join(directory, "config", "config.txt")
    os.makedirs(os.path.dirname(cfg), exist_ok=True)
    with open(cfg, "w") as f:
        f.write("D=3\nnp=1,1,1\n")
        f.write("X_start=" + ",".join(repr(float(v)) for v in w.x_start) + "\n")
        f.write(f"IMGname=data/{w.name}.raw\n")
        f.write(f"voxel_nb_X={nx}\nvoxel_nb_Y={ny}\nvoxel_nb_Z={nz}\n")
        f.write("ROI_start_X=0\nROI_start_Y=0\nROI_start_Z=0\n")
        f.write(f"voxel_size={w.voxel_size!r}\n")
        f.write("element_nb=" + ",".join(str(e) for e in w.element_nb) + "\n")
        for key, vals in (("u", w.mg_u), ("d", w.mg_d)):
            nu0, nu1, nu2, gamma, ncy = vals
            f.write(f"ncy_{key}={ncy}\nnu0_{key}={nu0}\nnu1_{key}={nu1}\nnu2_{key}={nu2}\ngamma_{key}={gamma}\n")
        f.write(f"lc={int(w.lc)}\n")
        for k, v in (extra or {}).items():
            f.write(f"{k}={v}\n")
    return {"raw": raw, "config": cfg}
