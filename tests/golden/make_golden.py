#!/usr/bin/env python3
"""Generates the golden fixtures of tests/golden/ from the REFERENCE itself.

The reference HPCrack sources are compiled as they are (oracle/Makefile -> oracle/_ref/
libhpcref.so, single-rank MPI stand-in) and driven through oracle/ref_harness.cpp on seeded
inputs; inputs and outputs are stored as compressed .npz fixtures.  The reference has no test
vectors of its own, so these are its golden vectors.  Run from the repository root:

    make -C oracle ref REF=<reference source tree> && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import bindings as B  # noqa: E402
from hpcrack_b200 import microstructure as ms  # noqa: E402
from cases import load_random  # noqa: E402

SMALL_K = 1e-5
LC = 2.0


def ops_case(ml, enb, x0, seed):
    """Single-operator outputs on random fields."""
    ref = B.RefOracle(ml, enb, x0=x0)
    data = load_random([ref], ml, enb, seed)
    out = {"ml": ml, "enb": np.array(enb), "x0": np.array(x0), "seed": seed}
    for l in range(ml + 1):
        f, ch, u, fu = data[l]
        for k, v in f.items():
            out[f"in_{k}_{l}"] = v
        out[f"in_choice_{l}"] = ch
        out[f"in_u_{l}"] = u
        out[f"in_fu_{l}"] = fu
    for l in range(ml + 1):
        ref.internal_force(l, B.U, B.RU, SMALL_K)
        out[f"if_{l}"] = ref.get(B.RU, l)
        ref.prem_u(l, B.RU, SMALL_K)
        out[f"prem_{l}"] = ref.get(B.RU, l)
        ref.fld(l, B.D, B.FD, LC)
        out[f"fld_{l}"] = ref.get(B.FD, l)
        ref.precondition_m(l, B.R, LC)
        out[f"pm_{l}"] = ref.get(B.R, l)
        ref.fd_h(l)
        out[f"fdh_{l}"] = ref.get(B.FD, l)
    # transfers of component 1 between the top two levels
    lf = ml
    if lf >= 1:
        ref.solution_injection(B.U, 1, lf)
        out["inject"] = ref.get(B.U, lf - 1)[1]
        ref.coarsen_f_standard(B.RU, B.FU, B.UOLD, 1, lf)
        out["restrict"] = ref.get(B.RU, lf - 1)[1]
        ref.set(B.UOLD, lf - 1, np.random.default_rng(seed + 1).standard_normal((3, ref.n(lf - 1))))
        out["in_uold"] = ref.get(B.UOLD, lf - 1)
        ref.refine_standard(B.FU, B.U, B.UOLD, 1, lf)
        out["prolong"] = ref.get(B.FU, lf)[1]
    # boundary conditions on the finest level
    ref.dirichlet_bd(ml, B.U, 0.37)
    out["bc_u"] = ref.get(B.U, ml)
    ref.dirichlet_force(ml, B.FU, B.U)
    out["bc_force"] = ref.get(B.FU, ml)
    ref.dirichlet_residual(ml, B.FU)
    out["bc_res"] = ref.get(B.FU, ml)
    # material selection and coarse element moduli (u is now the BC-adjusted field)
    ref.mp_choice()
    out["choice"] = ref.get_choice(ml)
    ref.mp_all_element(SMALL_K)
    out["ke"] = ref.get(B.KE, ml)
    out["ge"] = ref.get(B.GE, ml)
    ref.vr_all_level(B.KE)
    out["ke_vr"] = np.concatenate([ref.get(B.KE, l) for l in range(ml + 1)])
    ref.coarse_vr(B.GC)
    out["gc_vr"] = np.concatenate([ref.get(B.GC, l) for l in range(ml + 1)])
    ref.strain_history(LC, 3.5)
    out["H_hist"] = ref.get(B.H, ml)
    ref.voigt_all_level(B.H)
    out["H_voigt"] = np.concatenate([ref.get(B.H, l) for l in range(ml + 1)])
    out["ue"] = ref.U_e(LC)
    out["dmax"] = ref.d_max()
    out["ddmax"] = ref.delta_d_max()
    ref.externe_force_nodal(0.37, SMALL_K)
    out["reaction"] = ref.get(B.FU, ml)
    out["fsum"] = ref.externe_force_sum()
    ref.close()
    return out


def solver_case(seed):
    """Single smoother calls and one V-cycle of each kind on random fields, 17^3 over 9^3."""
    ml, enb = 1, (8, 8, 8)
    ref = B.RefOracle(ml, enb)
    load_random([ref], ml, enb, seed)
    out = {"ml": ml, "enb": np.array(enb), "seed": seed}
    it, fn = ref.pcg_u(1, SMALL_K, 1.0, 4, 0, 0.0)
    out["pcg_u_u"] = ref.get(B.U, 1)
    out["pcg_u_fnorm"] = fn
    it, fdn = ref.pcg_d(1, LC, 3, 0, 0.0)
    out["pcg_d_d"] = ref.get(B.D, 1)
    out["pcg_d_fdnorm"] = fdn
    ref.mp_all_element(SMALL_K)
    ref.vr_all_level(B.KE)
    ref.vr_all_level(B.GE)
    it, fn = ref.cycle_u(1, (50, 4, 2, 1, 12), SMALL_K, 1.0, 0, fn)
    out["cycle_u_u"] = ref.get(B.U, 1)
    out["cycle_u_fnorm"] = fn
    it, fdn = ref.cycle_d(1, (10, 2, 1, 1, 12), LC, 0, fdn)
    out["cycle_d_d"] = ref.get(B.D, 1)
    ref.close()
    return out


def steps_case(name, steps, reference_schedule, small_k=1e-5, mech_tol=1e-6, pf_tol=1e-12, keep=None):
    """Full staggered increments of a synthetic specimen, from the reference's own image and CSV
    input path; a pre-cracked workload gets its crack layer (H = H_crack on the crack elements, d = 1
    on their nodes, H Voigt-averaged to every level) before the first increment.  Fields are kept
    for the increments in `keep` (all by default); the step outputs for every increment.
    Tolerances other than the reference's own (1e-6, 1e-12) run through the harness driver that
    makes u_entire's / phase_field's calls with the threshold as a parameter."""
    import tempfile
    w = ms.make_workload(name)
    ref = B.RefOracle(w.maxlevel, w.element_nb, x0=w.x_start)
    with tempfile.TemporaryDirectory() as td:
        paths = ms.write_inputs(w, td)
        ref.input_total(td, paths["raw"], w.nodes, w.voxel_size)
    out = {"name": name, "steps": steps, "small_k": small_k, "mech_tol": mech_tol, "pf_tol": pf_tol}
    L = w.maxlevel
    if w.crack:
        Hc, dc = ms.precrack_fields(w)
        ref.set(B.H, L, Hc)
        ref.set(B.D, L, dc)
        ref.voigt_all_level(B.H)
    for f, key in ((B.BULK, "bulk"), (B.G, "g"), (B.GC, "gc")):
        out[key] = np.concatenate([ref.get(f, l) for l in range(L + 1)])
    kw = {} if reference_schedule else {"ut0": w.ut0, "dU": w.du}
    for t in range(steps):
        o = ref.step(t, w.mg_u, w.mg_d, small_k, w.lc, w.voxel_size, mech_tol=mech_tol, pf_tol=pf_tol, **kw)
        out[f"out_{t}"] = np.array(o)
        if keep is None or t in keep:
            out[f"u_{t}"] = ref.get(B.U, L)
            out[f"d_{t}"] = ref.get(B.D, L)
            out[f"H_{t}"] = ref.get(B.H, L)
    out["state"] = np.array(ref.state())
    ref.close()
    return out


def main():
    if not B.RefOracle.available():
        raise SystemExit("oracle/_ref/libhpcref.so missing: make -C oracle ref REF=<reference source tree>")
    B.RefOracle._load().ref_set_threads(os.cpu_count() or 1)
    builders = {
        "ops_iso": lambda: ops_case(2, (2, 2, 2), (-3.0, 1.5, -7.0), 11),
        "ops_xwide": lambda: ops_case(1, (4, 3, 2), (0.0, 0.0, 0.0), 12),
        "ops_ywide": lambda: ops_case(1, (2, 7, 3), (-1.0, -1.0, -1.0), 13),
        "solver": lambda: solver_case(21),
        "steps17": lambda: steps_case("small17", 4, reference_schedule=False),
        "steps17_ue": lambda: steps_case("small17", 2, reference_schedule=True),
        # the benchmarked specimen's recipe (three phases with pores, pre-crack) at 33^3: at the
        # benchmark's tolerance |r|/|f| <= 1e-8 (squared 1e-16) with fields of the first and last
        # increments, and at the reference's own thresholds (step outputs only)
        "crack33": lambda: steps_case("crack33", 3, reference_schedule=False, small_k=1e-6, mech_tol=1e-16,
                                      pf_tol=1e-16, keep=(0, 2)),
        "crack33_reftol": lambda: steps_case("crack33", 3, reference_schedule=False, small_k=1e-6, keep=()),
    }
    only = sys.argv[1:]  # optional subset of fixture names
    cases = {name: build() for name, build in builders.items() if not only or name in only}
    for name, data in cases.items():
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in data.items()})
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
