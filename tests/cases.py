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


# Pre-cracked specimens (the benchmarked recipe: pores, inclusions, a d = 1 crack layer).  The first
# increment is determined to rounding: every implementation agrees within 1e-10 with equal V-cycle
# counts.  From the second increment on the solve starts from the previous solution and the crack's
# residual stiffness (k = 1e-6) makes the displacement along the crack faces insensitive to the
# residual, so u is determined only to the rounding of the summation order: two runs of the
# reference itself on 8 OpenMP threads (whose element scatter order varies from run to run) differ
# on crack33 by 1.2e-9 to 4e-8 in u and by up to 1 V-cycle at |r|/|f| <= 1e-8, and by 1.1e-5 in u at
# the reference's own threshold |r|^2/|f|^2 <= 1e-6.  d and H do not depend on those modes and stay
# within 1e-14.  The bars below are those spreads with a margin of 25 or more.
CRACK_U_TOL = {1e-16: 1e-6, 1e-6: 1e-3}    # relative L2 of u from the second increment, by mech_tol
CRACK_F_TOL = {1e-16: 1e-9, 1e-6: 1e-5}    # relative difference of the reaction force
CRACK_CYCLE_SLACK = 1                      # V-cycles from the second increment


def crack_masks(w):
    """Element slots and nodes outside the pre-crack layer of a workload."""
    Hc, dc = ms.precrack_fields(w)
    return Hc == 0, dc == 0


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


def vtk_expected(option, values, dims, origin, spacing, filename, field_name, level, t, scale=1.0):
    """The .vti and .pvti bytes the reference's write_total_de ("S"), write_total_u ("V") and
    write_total_H ("C") produce for one rank (vtk_output.cpp:26-469), built independently from the
    file format: XML text, Float32 values x fastest (vector components interleaved, element slots
    for cell data), base64 of the 4-byte length header and of the values as two separate blocks.
    `values`: dense x-fastest doubles, shape (n,) or (3, n) for "V"."""
    import base64

    nx, ny, nz = dims
    ii, jj, kk = nx - 1, ny - 1, nz - 1
    if option == "V":
        v = np.asarray(values, dtype=np.float64).reshape(3, -1)
        data = (scale * v).T.astype(np.float32).ravel()
    elif option == "C":
        a = np.asarray(values, dtype=np.float64).reshape(nz, ny, nx)[:kk, :jj, :ii]
        data = a.astype(np.float32).ravel()
    else:
        data = np.asarray(values, dtype=np.float64).astype(np.float32).ravel()
    raw = data.astype("<f4").tobytes()
    hdr = base64.b64encode(np.uint32(len(raw)).astype("<u4").tobytes())
    x0, y0, z0 = origin
    hx, hy, hz = spacing
    head = ('<?xml version="1.0"?>\n'
            '<VTKFile type="ImageData" version="0.1" byte_order="LittleEndian">\n'
            f'<ImageData WholeExtent="0 {ii} 0 {jj} 0 {kk} " \t\t\t\tOrigin="{x0:f} {y0:f} {z0:f}" '
            f'Spacing="{hx:f} {hy:f} {hz:f}">\n'
            f'<Piece Extent="0 {ii} 0 {jj} 0 {kk}" >\n')
    ncomp = 3 if option == "V" else 1
    array = f'<DataArray Name="{field_name}" type="Float32" NumberOfComponents="{ncomp}" format="binary">\n'
    if option == "C":
        head += f'<PointData></PointData>\n<CellData Scalar = "{field_name}">\n' + array
        tail = "\n</DataArray>\n</CellData>\n"
    else:
        head += f'<PointData {"Vectors" if option == "V" else "Scalars"}="{field_name}">\n' + array
        tail = "\n</DataArray>\n</PointData>\n<CellData></CellData>\n"
    tail += "</Piece>\n</ImageData>\n</VTKFile>"
    vti = head.encode() + hdr + base64.b64encode(raw) + tail.encode()
    p = ('<?xml version="1.0"?>\n'
         '<VTKFile type="PImageData" version="0.1" byte_order="LittleEndian">\n'
         f'<PImageData WholeExtent="0 {ii} 0 {jj} 0 {kk} " \t\t\t\tGhostLevel="0" Origin="{x0:f} {y0:f} {z0:f}" '
         f'Spacing="{hx:f} {hy:f} {hz:f}">\n')
    parray = f'<PDataArray Name="{field_name}" type="Float32" NumberOfComponents="{ncomp}"/>\n'
    if option == "C":
        p += f'<PPointData></PPointData>\n<PCellData Scalar = "{field_name}">\n' + parray + "</PCellData>\n"
    else:
        p += f'<PPointData {"Vectors" if option == "V" else "Scalars"}="{field_name}">\n' + parray
        p += "</PPointData>\n<PCellData></PCellData>\n"
    p += (f'<Piece Extent="0 {ii} 0 {jj} 0 {kk}" Source="{filename}_l_{level}_t_{t}_Proc_0.vti"/>\n'
          "</PImageData>\n</VTKFile>\n")
    return vti, p.encode()


def vtk_paths(workdir, filename, level, t):
    import os

    return (os.path.join(workdir, "Output", f"{filename}_l_{level}_t_{t}_Proc_0.vti"),
            os.path.join(workdir, "Output", f"{filename}_l_{level}_t_{t}.pvti"))
