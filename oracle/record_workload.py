"""Record the FP64 CG iteration count of the benchmark workload -- TEST
INFRASTRUCTURE ONLY.

Solves the 32^3x64 workload (seeded U = exp(i 0.25 H) links, one Gaussian
source, kappa 0.16, mu 0.005, antiperiodic T) once, in full, with the
reference's CG (physics/algorithms/solvers/cg.cpp:277-400 restated in
c2q_oracle.c) on the reference's own kernels compiled as C (the "reference"
oracle build; the restatement of the kernels where that build is absent), with
the reference's stopping test |r|^2 < prec, prec = (1e-10)^2 |b|^2, checked every
10 iterations.  Writes oracle/workload_fp64_cg.json: the parameters, the
iterations the solve performed, its true residual and its wall time.

The CPU reference arm of bench.py times a bounded number of these iterations
per step and scales by the recorded count; the GPU tests check that the
library's FP64 CG with the same stopping test needs the same count.

    python oracle/record_workload.py        (a few minutes on 8 cores)
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402

WORKLOAD = {"ns": 32, "nt": 64, "eps": 0.25, "kappa": 0.16, "mu": 0.005, "gauge_seed": 20250,
            "source_seed": 777, "source": "gaussian", "theta_t": 1.0, "theta_s": 0.0, "rel_tol": 1e-10,
            "operator": "QplusQminus_eo"}
OUT = os.path.join(HERE, "workload_fp64_cg.json")


def main():
    w = WORKLOAD
    kind = "reference" if O.available("reference") else "port"
    o = O.Oracle(kind)
    o.set_lattice(w["ns"], w["nt"], w["theta_t"], w["theta_s"])
    g = o.gauge_generate(w["ns"], w["nt"], w["eps"], w["gauge_seed"])
    b = o.source_generate(o.seo, w["source"], w["source_seed"])
    b2 = float((b * b).sum())
    mubar = 2 * w["kappa"] * w["mu"]
    x = np.zeros_like(b)
    P = O.SolverParams(prec=w["rel_tol"] ** 2 * b2, cgmax=10000, solver=1)
    t0 = time.perf_counter()
    ret = o.cg(x, O.OP_QPQM_EO, b, g, w["kappa"], mubar, params=P)
    sec = time.perf_counter() - t0
    if ret < 0:
        raise SystemExit(f"reference CG failed with status {ret}")
    r = o.apply(O.OP_QPQM_EO, x, g, w["kappa"], mubar) - b
    rec = {"workload": w, "oracle": kind, "cg_returned": int(ret),
           "iterations": int(ret) + 1,  # the reference's cg returns the index of its last iteration
           "true_resid_rel": float(np.linalg.norm(r) / np.sqrt(b2)), "seconds": round(sec, 1),
           "threads": int(os.environ.get("OMP_NUM_THREADS", "0")) or os.cpu_count(),
           "made_by": "python oracle/record_workload.py"}
    with open(OUT, "w") as f:
        json.dump(rec, f, indent=1)
        f.write("\n")
    print(json.dumps(rec))


if __name__ == "__main__":
    main()
