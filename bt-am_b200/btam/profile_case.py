"""Fixed-shape evaluation runs for kernel profiling.

Builds one synthetic system, pins the launch variants (no autotuner, so the
launch sequence is known in advance) and runs a few residual evaluations in
one arithmetic form.  Meant to run under a profiler with a kernel filter and
a launch count, e.g.

    ncu --set full --clock-control none -k regex:pass2u_pair -s 2 -c 1 \\
        python -m btam.profile_case --workload dropin --precision fp32c

(from bt-am_b200/, or with bt-am_b200 on PYTHONPATH).

With --stretch the run is one bulk stretch relaxation (the non-mean-field
point kernels) instead of the evaluations.

Workloads: "dropin" is the plain drop-in system (periodic hcp Mg 20x15x15
hexagonal cells with H on all tetrahedral sites, 27 000 sites); "small" is a
periodic ortho-hexagonal block of about 1 500 Mg with H on 30 % of the
tetrahedral sites, for quick captures.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import btam
from btam import lattice


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="dropin", choices=["dropin", "small"])
    ap.add_argument("--precision", default="fp32c", choices=["fp32c", "fp64"])
    ap.add_argument("--v1", type=int, default=None, help="pass-1 variant (default: 19 fp32c, 25 fp64)")
    ap.add_argument("--v2", type=int, default=None, help="pass-2 variant (default: 27 fp32c, 25 fp64)")
    ap.add_argument("--evals", type=int, default=4)
    ap.add_argument("--stretch", action="store_true",
                    help="run the bulk stretch relaxation (non-mean-field forms) instead")
    ap.add_argument("--multipole", type=int, default=0, choices=[0, 1, 2],
                    help="evaluate rho-bar and V0 under the multipole rule (1: FD Hessians, "
                         "2: analytic) instead")
    ap.add_argument("--residuals", action="store_true",
                    help="with --multipole: the residuals instead of rho-bar and V0")
    args = ap.parse_args()
    prec = btam.FP32C if args.precision == "fp32c" else btam.FP64
    if args.workload == "dropin":
        sysd = lattice.config2()
    else:
        sysd = lattice.periodic_cube(1500, seed=1)
    tables = btam.Tables()
    S = btam.System(tables, sysd)
    S.build_neighbors()
    if args.multipole:
        fn = S.mf_residuals_multipole if args.residuals else S.mf_eval_multipole
        fn(args.multipole)  # warm-up
        t0 = time.perf_counter()
        for _ in range(args.evals):
            res = fn(args.multipole)
        dt = time.perf_counter() - t0
        nr, ng, npairs = S.info()
        print(json.dumps({"workload": args.workload, "multipole_rule": args.multipole,
                          "what": "residuals" if args.residuals else "rho, V0",
                          "sites": nr, "pairs": npairs, "evals": args.evals,
                          "wall_ms_per_eval": dt * 1e3 / args.evals,
                          "finite": bool(all(np.isfinite(r).all() for r in res[:2]))}))
        S.close()
        tables.close()
        return
    if args.stretch:
        t0 = time.perf_counter()
        F, info = S.relax_stretch(atol=1e-12, rtol=1e-10, max_iter=20)
        dt = time.perf_counter() - t0
        print(json.dumps({"workload": args.workload, "stretch": [float(f) for f in F],
                          "residual_evaluations": info["evaluations"], "norm": info["norm"],
                          "status": info["status"], "wall_ms": dt * 1e3}))
        S.close()
        tables.close()
        return
    v1 = args.v1 if args.v1 is not None else (19 if prec == btam.FP32C else 25)
    v2 = args.v2 if args.v2 is not None else (27 if prec == btam.FP32C else 25)
    S.set_variants(prec, v1, v2)
    t0 = time.perf_counter()
    for _ in range(args.evals):
        S.evaluate_async(prec)
    S.sync()
    dt = time.perf_counter() - t0
    tot = S.results(want=("totals",))["totals"]
    nr, ng, npairs = S.info()
    print(json.dumps({"workload": args.workload, "precision": args.precision, "v1": v1, "v2": v2,
                      "sites": nr, "images": ng, "pairs": npairs, "evals": args.evals,
                      "wall_ms_per_eval": dt * 1e3 / args.evals,
                      "energy": float(tot[0]), "finite": bool(np.isfinite(tot).all())}))
    S.close()
    tables.close()


if __name__ == "__main__":
    main()
