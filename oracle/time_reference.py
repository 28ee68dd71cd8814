"""Times the reference's own CPU code (oracle/_ref, compiled from its sources) on full staggered
increments of a synthetic workload: 1 rank x every host core as OpenMP threads, at the reference's
own thresholds (|r|^2/|f|^2 <= 1e-6 mechanical, |R|^2/|fd|^2 <= 1e-12 phase field).  Test
infrastructure: the CPU baseline beside the library, never part of it.

    python -m oracle.time_reference parity129 3      # one JSON line per increment, then a summary
"""
import json
import os
import sys
import tempfile
import time


def main(argv):
    name = argv[1] if len(argv) > 1 else "parity65"
    steps = int(argv[2]) if len(argv) > 2 else 3
    from hpcrack_b200 import microstructure as ms
    from hpcrack_b200.solver import D, H
    from oracle import bindings as B

    cores = os.cpu_count() or 1
    B.RefOracle._load().ref_set_threads(cores)
    w = ms.make_workload(name)
    ref = B.RefOracle(w.maxlevel, w.element_nb, x0=w.x_start)
    with tempfile.TemporaryDirectory() as td:
        paths = ms.write_inputs(w, td)
        t0 = time.perf_counter()
        ref.input_total(td, paths["raw"], w.nodes, w.voxel_size)
        t_in = time.perf_counter() - t0
    if w.crack:
        Hc, dc = ms.precrack_fields(w)
        ref.set(H, w.maxlevel, Hc)
        ref.set(D, w.maxlevel, dc)
        ref.voigt_all_level(H)
    nx, ny, nz = w.nodes
    n = nx * ny * nz
    total_s, work = 0.0, 0.0
    cycles = []
    for t in range(steps):
        t0 = time.perf_counter()
        o = ref.step(t, w.mg_u, w.mg_d, w.small_k, w.lc, w.voxel_size, ut0=w.ut0, dU=w.du)
        dt = time.perf_counter() - t0
        total_s += dt
        work += 3.0 * n * o[6] + n * o[7]
        cycles.append((int(o[4]), int(o[5])))
        print(json.dumps({"t": t, "s": dt, "mech_cycles": int(o[4]), "pf_cycles": int(o[5]),
                          "mech_iters": int(o[6]), "pf_iters": int(o[7]), "F": o[1]}), flush=True)
    ref.close()
    print(json.dumps({"workload": name, "nodes": n, "increments": steps, "cores": cores,
                      "layout": f"1 rank x {cores} OpenMP threads", "input_total_s": t_in, "total_s": total_s,
                      "mdof_iter_per_s": work / total_s / 1e6 if total_s > 0 else None,
                      "s_per_v_cycle": total_s / max(1, sum(a + b for a, b in cycles)), "v_cycles": cycles}),
          flush=True)


if __name__ == "__main__":
    main(sys.argv)
