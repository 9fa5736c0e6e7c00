"""Benchmark: tm-Wilson eo CG solves/s to a true residual of 1e-10 on 32^3x64.

One step = one complete CG solve (QplusQminus_eo, kappa 0.16, mu 0.005,
antiperiodic T, gauge U = exp(i 0.25 H), one Gaussian source) from x = 0 to
||b - A x|| / ||b|| <= 1e-10 checked in FP64.  The headline `value` is the
mixed-precision solver (FP16 fixed-point spinors and 12-real FP16 links in the
inner CG, FP32 arithmetic, FP64 reliable updates); the plain FP64 solver on the
same problem is reported beside it.  `value` is device time with inputs
resident in HBM; `e2e` goes through the public API with pinned host buffers
(source upload, solve, solution download) inside the timed region.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
For N > 1 (torchrun) each rank solves its own replica on its own GPU (the path
does not shard); value = all ranks' solves / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "tm-Wilson CG solves/s @1e-10 (mixed vs FP64, same B200); Dslash HBM GB/s; p99"
NS, NT = 32, 64
EPS, KAPPA, MU = 0.25, 0.16, 0.005
GAUGE_SEED, SOURCE_SEED = 20250, 777
REL_TOL = 1e-10
# The FP64 CG iterations the reference's CG (on its own kernels, with its stopping
# test |r|^2 < REL_TOL^2 |b|^2) performed on this workload, recorded by one full
# CPU solve (oracle/record_workload.py); the CPU arm times a bounded sample of
# those iterations and scales by this count.
WORKLOAD_RECORD = os.path.join(ROOT, "oracle", "workload_fp64_cg.json")
WORKLOAD = (f"32^3x64 tm-Wilson eo CG on QplusQminus_eo, 1 gaussian source, kappa {KAPPA}, mu {MU}, "
            f"eps {EPS}, antiperiodic T, x0 = 0, true residual {REL_TOL}")


def bench_config(ws, precision=16):
    """The `config` of the JSON line, the same for the GPU and the reference arm."""
    return {"workload": WORKLOAD, "lattice": "32x32x32x64", "global_batch": ws,
            "inner_precision": precision, "links": "12-real", "parallelism": f"replicas x{ws}",
            "l2": "inputs larger than L2 (FP16 12-real links 201 MB, FP64 links 1.2 GB)"}


def recorded_fp64_iterations():
    """(iterations, record) of the reference's FP64 CG on this workload, or (None, why)."""
    try:
        with open(WORKLOAD_RECORD) as f:
            rec = json.load(f)
    except OSError as e:
        return None, f"no recorded FP64 iteration count ({e.strerror})"
    w = rec["workload"]
    if (w["ns"], w["nt"], w["eps"], w["kappa"], w["mu"], w["gauge_seed"], w["source_seed"], w["rel_tol"]) != \
            (NS, NT, EPS, KAPPA, MU, GAUGE_SEED, SOURCE_SEED, REL_TOL):
        return None, "the recorded FP64 iteration count is for another workload"
    return int(rec["iterations"]), rec


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", type=int, default=16, choices=[16, 32, 64])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-large", action="store_true", help="skip the 64^3x128 (config 5) section of the default run")
    ap.add_argument("--serve", action="store_true",
                    help="serving sweep only: Poisson requests at rising rates, p50/p99 latency and solves/s")
    ap.add_argument("--serve-requests", type=int, default=16)
    ap.add_argument("--serve-rates", default="0.5,1,2,4")
    ap.add_argument("--serve-slots", default="4",
                    help="comma-separated slot counts; the same request list is served with each")
    ap.add_argument("--phase", default="all", choices=["all", "mixed", "dslash", "large", "mrhs"],
                    help="mixed: only the warm-up and timed mixed-precision solves (for profiling); "
                         "mrhs: batched multi-RHS solves on --ns^3 x --nt (for profiling a batched sweep)")
    ap.add_argument("--ns", type=int, default=24)
    ap.add_argument("--nt", type=int, default=48)
    ap.add_argument("--nrhs", type=int, default=12)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def mbar():
    return 2.0 * KAPPA * MU


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM traffic of the dominant sweep from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
            return
        # wait until the sampler produces rows, so the timed region is covered
        t0 = time.time()
        while time.time() - t0 < 5.0:
            self.f.flush()
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        def num(v):
            try:
                return float(v)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": num(rows[0][2]),
                "reasons": sorted(reasons), "samples": len(rows)}


# ------------------------------------------------------------------ CPU reference arm
def cpu_reference_sample(g, b, fp64_iters, budget_s=15.0):
    """Time the reference's own kernels (oracle/_ref, compiled from the reference
    sources) running the reference CG on this workload for a bounded number of
    iterations, and scale to solves/s with the FP64 iteration count."""
    import oracle as O
    kind = "reference" if O.available("reference") else "port"
    o = O.Oracle(kind)
    o.set_lattice(NS, NT, 1.0, 0.0)
    threads = int(os.environ.get("OMP_NUM_THREADS", "0")) or os.cpu_count()
    x = np.zeros_like(b)
    P = O.SolverParams(prec=1e-300, cgmax=1, solver=1)
    t0 = time.perf_counter()
    o.cg(x, O.OP_QPQM_EO, b, g, KAPPA, mbar(), params=P)  # refresh + 1 iteration
    t1 = time.perf_counter() - t0
    n = max(1, min(40, int(budget_s / max(t1, 1e-3) * 2) - 1))
    x[:] = 0
    P = O.SolverParams(prec=1e-300, cgmax=n, solver=1)
    t0 = time.perf_counter()
    o.cg(x, O.OP_QPQM_EO, b, g, KAPPA, mbar(), params=P)
    tn = time.perf_counter() - t0
    # n iterations + one refresh (one extra operator application and saxpy)
    per_iter = tn / (n + 1)
    solves = 1.0 / (per_iter * fp64_iters)
    return {"value": solves, "unit": "solves/s", "cores": threads, "kind": kind,
            "sample": f"{n} FP64 CG iterations (+1 refresh) of this 32^3x64 workload on the reference's kernels "
                      f"in {tn:.1f} s; solves/s = 1 / (seconds per iteration x {fp64_iters}), the iterations the "
                      f"reference's CG performed in a full solve of this workload (oracle/workload_fp64_cg.json)",
            "seconds_per_iteration": per_iter}


def cpu_reference_extras(g, b, budget_s=10.0):
    """Beside the solve-rate sample: the reference's dslash_eo on the host cores in
    GB/s by the algorithmic byte model (1536 B/site, FP64 18-real), and config 1
    (8^4, eps 0.3, kappa 0.15, mu 0.01, one Z2 source) solved to a true residual
    1e-10 by the reference CG on its own kernels."""
    import oracle as O
    kind = "reference" if O.available("reference") else "port"
    o = O.Oracle(kind)
    o.set_lattice(NS, NT, 1.0, 0.0)
    o.dslash_eo(b, g, O.ODD, KAPPA)  # warm-up
    n, t0 = 0, time.perf_counter()
    while n < 3 and (n == 0 or time.perf_counter() - t0 < budget_s):
        o.dslash_eo(b, g, O.ODD, KAPPA)
        n += 1
    t = time.perf_counter() - t0
    gbs = DSLASH_BYTES[(64, 0)] * b.shape[0] * n / t / 1e9
    o.set_lattice(8, 8, 1.0, 0.0)
    c1 = {"g": o.gauge_generate(8, 8, 0.3, 1), "b": o.source_generate(o.seo, "z2", 2)}
    b2 = float((c1["b"] ** 2).sum())
    P = O.SolverParams(prec=REL_TOL ** 2 * b2, cgmax=10000, solver=1)
    x = np.zeros_like(c1["b"])
    o.cg(x, O.OP_QPQM_EO, c1["b"], c1["g"], 0.15, 2 * 0.15 * 0.01, params=P)  # warm-up
    m, t0 = 0, time.perf_counter()
    while m < 20 and (m == 0 or time.perf_counter() - t0 < budget_s):
        x[:] = 0
        o.cg(x, O.OP_QPQM_EO, c1["b"], c1["g"], 0.15, 2 * 0.15 * 0.01, params=P)
        m += 1
    t1 = time.perf_counter() - t0
    o.set_lattice(NS, NT, 1.0, 0.0)
    return {"dslash_gbs": round(gbs, 2), "dslash_sample": f"{n} FP64 18-real dslash_eo sweeps of 32^3x64",
            "config1_solves_per_s": round(m / t1, 2), "config1_sample": f"{m} solves of 8^4 to 1e-10"}


def oracle_check(g, b, x, ms_precision):
    """The benchmark's final mixed-precision solution checked by the oracle:
    ||b - A x|| / ||b|| recomputed on the host by the reference's own kernels
    with the 18-real FP64 links as generated (outside every timed region)."""
    import oracle as O
    kind = "reference" if O.available("reference") else "port"
    o = O.Oracle(kind)
    o.set_lattice(NS, NT, 1.0, 0.0)
    t0 = time.perf_counter()
    r = o.apply(O.OP_QPQM_EO, x, g, KAPPA, mbar())
    r -= b
    rel = float(np.linalg.norm(r) / np.linalg.norm(b))
    return {"true_resid_rel": rel, "pass": rel <= REL_TOL * (1 + 1e-6), "oracle": kind,
            "operator": "QplusQminus_eo on the 18-real FP64 links as generated",
            "solution": f"the last timed mixed-precision (FP{ms_precision} inner) solve",
            "seconds": round(time.perf_counter() - t0, 2)}


def config1_inputs(c2q):
    """config 1: 8^4, eps 0.3 links, one Z2 source (kappa 0.15, mu 0.01)."""
    lat = c2q.Lattice(8, 8, 1.0, 0.0)
    return {"lat": lat, "g": c2q.host.generate_gaugefield(lat, 0.3, 1),
            "b": c2q.host.generate_source(lat.seo, "z2", 2)}


def config1_gpu(c2q, system, e0, e1, n=20):
    """config 1 on the GPU: FP64 eo CG (the reference's algorithm) to a true residual 1e-10,
    its iterations replayed as a CUDA graph (the lattice is too small to hide launches)."""
    import torch
    c1 = config1_inputs(c2q)
    gf = c2q.Gaugefield(system, c1["lat"], c1["g"])
    B = c2q.Spinorfield_eo(system, c1["lat"], c1["b"])
    X = c2q.Spinorfield_eo(system, c1["lat"])
    add = c2q.AdditionalParameters(0.15, 2 * 0.15 * 0.01)
    A = c2q.host.QplusQminus_eo()
    P = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=10000, precision=64, use_graph=True)
    rep = {}
    for _ in range(3):
        X.zero()
        c2q.host.cg(X, A, gf, B, P, add, rep)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(n):
        X.zero()
        c2q.host.cg(X, A, gf, B, P, add)
    e1.record()
    torch.cuda.synchronize()
    return {"workload": "8^4, eps 0.3, kappa 0.15, mu 0.01, one Z2 source, FP64 eo CG to 1e-10",
            "gpu_fp64_solves_per_s": round(n / (e0.elapsed_time(e1) / 1e3), 1),
            "iterations": rep["iterations"], "true_resid_rel": rep["true_resid_rel"]}


# algorithmic bytes per site of one plain dslash_eo sweep: 8 links + input + output
DSLASH_BYTES = {(64, 0): 8 * 144 + 2 * 192, (64, 1): 8 * 96 + 2 * 192, (32, 0): 8 * 72 + 2 * 96,
                (32, 1): 8 * 48 + 2 * 96, (16, 1): 8 * 24 + 2 * 52}


def dslash_gbs(c2q, system, lat, gf, b, e0, e1, n=20):
    """Achieved GB/s of c2q_dslash_eo (the public call) per storage precision and
    link format, from CUDA events around n launches on the library's stream."""
    import torch
    lib = system.lib
    out = {}
    for (prec, rec12), per_site in DSLASH_BYTES.items():
        system.set_link_format(rec12)
        A_ = c2q.Spinorfield_eo(system, lat, b, precision=prec)
        Y_ = c2q.Spinorfield_eo(system, lat, precision=prec)
        for _ in range(3):
            lib.c2q_dslash_eo(Y_.h, gf.h, A_.h, 1, KAPPA)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            lib.c2q_dslash_eo(Y_.h, gf.h, A_.h, 1, KAPPA)
        e1.record()
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3 / n
        out[f"fp{prec}_{12 if rec12 else 18}real"] = {"gbs": round(lat.seo * per_site / sec / 1e9, 1),
                                                     "us": round(sec * 1e6, 1), "bytes_per_site": per_site}
        del A_, Y_
    system.set_link_format(False)
    return out


def large_volume(c2q, system, e0, e1, bicgstab_cgmax=2000, oracle_check_solution=False):
    """64^3x128 (16.8 M eo sites), eps 0.2, kappa 0.1625, mu 0.003, one Gaussian
    source: dslash GB/s per precision (FP64 gauge 18-real vs 12-real) and the
    solve time to a true residual 1e-10 of FP64 CG, FP64 BiCGStab (on Aee; it does
    not converge on this operator, nor does the reference's, so it is bounded by
    bicgstab_cgmax) and mixed-precision CG (FP16 / FP32 inner); each CG timed on its
    second solve.  With oracle_check_solution the mixed FP16 solution's true
    residual is recomputed by the oracle (the reference's kernels on the host)."""
    import torch
    ns, nt, kappa, mu = 64, 128, 0.1625, 0.003
    lat = c2q.Lattice(ns, nt, 1.0, 0.0)
    t = time.time()
    g = c2q.host.generate_gaugefield(lat, 0.2, 64128)
    gf = c2q.Gaugefield(system, lat, g)
    if not oracle_check_solution:
        del g
    b = c2q.host.generate_source(lat.seo, "gaussian", 128)
    setup_s = time.time() - t
    out = {"lattice": "64^3x128", "eo_sites": lat.seo, "kappa": kappa, "mu": mu, "eps": 0.2,
           "setup_s": round(setup_s, 1), "dslash_gbs": dslash_gbs(c2q, system, lat, gf, b, e0, e1, n=5)}
    add = c2q.AdditionalParameters(kappa, 2 * kappa * mu)
    B = c2q.Spinorfield_eo(system, lat, b)
    X = c2q.Spinorfield_eo(system, lat)
    b2 = float(np.vdot(b.reshape(-1), b.reshape(-1)))
    runs = {
        "fp64_cg": (c2q.host.cg, c2q.host.QplusQminus_eo(),
                    c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=40000, precision=64)),
        # the reference's BiCGStab "save" variant (true-residual recheck), bounded
        "fp64_bicgstab_save": (c2q.host.bicgstab, c2q.host.Aee(),
                               c2q.SolverParameters(solver="bicgstab_save", prec=REL_TOL ** 2 * b2,
                                                    cgmax=bicgstab_cgmax)),
        "mixed_fp16_cg": (c2q.host.cg, c2q.host.QplusQminus_eo(),
                          c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=40000, precision=16,
                                               use_rec12=True, use_graph=True)),
        "mixed_fp32_cg": (c2q.host.cg, c2q.host.QplusQminus_eo(),
                          c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=40000, precision=32,
                                               use_rec12=True, use_graph=True)),
    }
    sols = {}
    for name, (fn, A_, P_) in runs.items():
        if name != "fp64_bicgstab_save":  # one untimed solve first: pools, autotuner, derived links
            X.zero()
            fn(X, A_, gf, B, P_, add, {})
        X.zero()
        rep = {}
        torch.cuda.synchronize()
        e0.record()
        try:
            fn(X, A_, gf, B, P_, add, rep)
            ok = True
        except Exception as e:  # reported, not fatal
            ok = repr(e)
        e1.record()
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        x = X.dump()
        # true residual of the eo system the solver was given, in FP64 through the public operator
        R = c2q.Spinorfield_eo(system, lat)
        A_(R, gf, X, add)
        r = R.dump() - b
        out[name] = {"seconds": round(sec, 3), "iterations": rep.get("iterations"),
                     "reliable_updates": rep.get("reliable_updates"), "ok": ok,
                     "true_resid_rel": float(np.linalg.norm(r) / np.sqrt(b2))}
        sols[name] = x
        del R
    ref = sols["fp64_cg"]
    for name in ("mixed_fp16_cg", "mixed_fp32_cg"):
        out[name]["rel_err_vs_fp64_cg"] = float(np.linalg.norm(sols[name] - ref) / np.linalg.norm(ref))
    out["speedup_mixed_fp16_vs_fp64_cg"] = out["fp64_cg"]["seconds"] / out["mixed_fp16_cg"]["seconds"]
    if oracle_check_solution:
        import oracle as O
        kind = "reference" if O.available("reference") else "port"
        o = O.Oracle(kind)
        o.set_lattice(ns, nt, 1.0, 0.0)
        r = o.apply(O.OP_QPQM_EO, sols["mixed_fp16_cg"], g, kappa, 2 * kappa * mu)
        r -= b
        rel = float(np.linalg.norm(r) / np.sqrt(b2))
        out["oracle_check"] = {"solution": "mixed_fp16_cg", "true_resid_rel": rel, "pass": rel <= REL_TOL * (1 + 1e-6),
                               "oracle": kind, "operator": "QplusQminus_eo on the 18-real FP64 links as generated"}
        del g, r
    return out


def mrhs_phase(c2q, args):
    """Profiling driver of the batched sweeps: on ns^3 x nt (default 24^3 x 48,
    whose fields and links together exceed L2), kappa 0.16, mu 0.005, eps 0.25
    links, nrhs spin-colour point sources solved by the mixed-precision CG with
    FP16 inner fields, once as one batch and once one source at a time, without
    graphs, with a fixed launch configuration (no autotuner launches); reports
    the per-launch time of the inner sweeps of each."""
    import torch
    os.environ["C2Q_AUTOTUNE"] = "0"
    system = c2q.System(0)
    lat = c2q.Lattice(args.ns, args.nt, 1.0, 0.0)
    gf = c2q.Gaugefield(system, lat, c2q.host.generate_gaugefield(lat, EPS, GAUGE_SEED))
    add = c2q.AdditionalParameters(KAPPA, mbar())
    A = c2q.host.QplusQminus_eo()
    n = args.nrhs
    Bs = [c2q.Spinorfield_eo(system, lat, c2q.host.point_source(lat.seo, k % 12)) for k in range(n)]
    Xs = [c2q.Spinorfield_eo(system, lat) for _ in range(n)]
    P = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=40000, precision=16, use_rec12=True)
    out = {"lattice": f"{args.ns}^3x{args.nt}", "nrhs": n}
    lib = system.lib
    for label, batches in (("batch", [list(range(n))]), ("single", [[k] for k in range(n)])):
        for x_ in Xs:
            x_.zero()
        lib.c2q_ctx_profile(system.h, 1)
        t0 = time.perf_counter()
        for bt in batches:
            c2q.host.cg_multi([Xs[k] for k in bt], A, gf, [Bs[k] for k in bt], P, add)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        nl, ms, by = C.c_longlong(), C.c_double(), C.c_double()
        lib.c2q_ctx_profile_read(system.h, 16, C.byref(nl), C.byref(ms), C.byref(by))
        lib.c2q_ctx_profile(system.h, 0)
        out[label] = {"sweeps": nl.value, "sweep_ms_total": round(ms.value, 3), "solve_wall_s": round(wall, 3),
                      "sweep_gbs": round(by.value / (ms.value * 1e-3) / 1e9, 1) if ms.value > 0 else None}
    out["per_rhs_sweep_time_batch_over_single"] = out["batch"]["sweep_ms_total"] / out["single"]["sweep_ms_total"]
    system.close()
    return out


SERVE_VOLUMES = [(16, 32), (24, 48), (32, 64), (48, 96)]


def serving_run(c2q, rates, n_requests, slots=4, seed=4242, log=None, max_heavy=1):
    """Poisson-arriving inversion requests: volume uniform over SERVE_VOLUMES
    (one resident gauge field per volume, eps ~ U[0.2, 0.35]), kappa ~ U[0.14, 0.16],
    mu ~ U[0.002, 0.02], 1-12 Z2 sources, mixed-precision (FP16 inner) to 1e-10.
    The request list and the unit-rate arrival gaps are drawn once, so every
    rate serves the same requests and only the arrival spacing changes.
    For each arrival rate: latency = completion - submission per request,
    p50 / p99 (nearest rank), and solves/s = sources solved / wall time."""
    rng = np.random.default_rng(seed)
    server = c2q.host.Server(0, slots=slots, precision=16)
    server.set_heavy_limit(1 << 19, max_heavy)
    lats = []
    t_setup = time.time()
    for v, (ns, nt) in enumerate(SERVE_VOLUMES):
        lat = c2q.Lattice(ns, nt, 1.0, 0.0)
        g = c2q.host.generate_gaugefield(lat, float(rng.uniform(0.2, 0.35)), 9000 + v)
        server.add_gauge(v, lat, g)
        del g
        lats.append(lat)
    t_setup = time.time() - t_setup
    P = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=40000)
    out = {"volumes": [f"{ns}^3x{nt}" for ns, nt in SERVE_VOLUMES], "slots": slots, "inner_precision": 16,
           "heavy_requests_at_a_time": max_heavy, "heavy": "eo sites x sources >= 2^19",
           "sources": "Z2, 1-12 per request", "gauge_setup_s": round(t_setup, 1),
           "budget_bytes": server.stats()["budget_bytes"], "gauge_bytes": server.stats()["gauge_bytes"],
           "rates": []}
    reqs = [(int(rng.integers(0, len(SERVE_VOLUMES))), float(rng.uniform(0.14, 0.16)),
             float(rng.uniform(0.002, 0.02)), int(rng.integers(1, 13)), int(rng.integers(1, 1 << 40)))
            for _ in range(n_requests)]
    unit_gaps = rng.exponential(1.0, n_requests)
    for rate in rates:
        gaps = unit_gaps / rate
        t0 = time.time()
        tickets, next_t = [], 0.0
        for gap, (v, kappa, mu, n, sd) in zip(gaps, reqs):
            next_t += gap
            dt = t0 + next_t - time.time()
            if dt > 0:
                time.sleep(dt)
            tickets.append(server.submit(lats[v], v, kappa, mu, n, sd, params=P))
        res = [server.wait(t) for t in tickets]
        wall = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
        lat_s = sorted(r["t_done"] - r["t_submit"] for r in res)
        q = lambda f: lat_s[min(len(lat_s) - 1, int(np.ceil(f * len(lat_s))) - 1)]
        nsolved = sum(r["nsrc"] for r in res if r["status"] == 0)
        entry = {"rate_per_s": rate, "requests": n_requests, "p50_s": round(q(0.5), 4), "p99_s": round(q(0.99), 4),
                 "mean_s": round(float(np.mean(lat_s)), 4), "solves_per_s": round(nsolved / wall, 2),
                 "requests_per_s": round(n_requests / wall, 3), "failed": sum(r["status"] != 0 for r in res),
                 "true_resid_rel_max": max(r["true_resid_rel_max"] for r in res),
                 "iterations_max": max(r["iterations_max"] for r in res),
                 "queue_wait_mean_s": round(float(np.mean([r["t_admit"] - r["t_submit"] for r in res])), 4)}
        out["rates"].append(entry)
        if log:
            log(entry)
    server.close()
    return out


def inputs():
    import cl2qcd_b200 as c2q
    lat = c2q.Lattice(NS, NT, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(lat, EPS, GAUGE_SEED)
    b = c2q.host.generate_source(lat.seo, "gaussian", SOURCE_SEED)
    return lat, g, b


def run_reference(args, budget_s=150.0):
    """The reference arm: the reference's own kernels (oracle/_ref, compiled from
    the reference sources; the restatement if they are absent) running the
    reference CG on this workload on the host cores, with the workload's inputs
    from the oracle's own generators (bit-identical to the library's; the
    library is not loaded).  args.warmup untimed and args.steps timed steps;
    each step is one CG call of a bounded number of iterations, sized so the
    whole run takes about budget_s; solves/s scales the measured time per
    iteration by the iteration count the reference's CG needed for a full solve
    of this workload (recorded by oracle/record_workload.py).  Under torchrun
    only rank 0 runs."""
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    iters, rec = recorded_fp64_iterations()
    if iters is None:
        print(json.dumps({"impl": "reference", "unavailable": rec}))
        return 0
    import oracle as O
    kind = "reference" if O.available("reference") else "port"
    o = O.Oracle(kind)
    o.set_lattice(NS, NT, 1.0, 0.0)
    g = o.gauge_generate(NS, NT, EPS, GAUGE_SEED)
    b = o.source_generate(o.seo, "gaussian", SOURCE_SEED)
    threads = int(os.environ.get("OMP_NUM_THREADS", "0")) or os.cpu_count()
    x = np.zeros_like(b)

    def step(n):  # one CG call: a refresh and n iterations
        x[:] = 0
        o.cg(x, O.OP_QPQM_EO, b, g, KAPPA, mbar(), params=O.SolverParams(prec=1e-300, cgmax=n, solver=1))

    t0 = time.perf_counter()
    step(1)
    t_iter = (time.perf_counter() - t0) / 2
    steps, warmup = max(1, args.steps), max(0, args.warmup)
    n = max(1, min(40, int(budget_s / (steps + warmup) / max(t_iter, 1e-3)) - 1))
    for _ in range(warmup):
        step(n)
    t0 = time.perf_counter()
    for _ in range(steps):
        step(n)
    t = time.perf_counter() - t0
    per_iter = t / (steps * (n + 1))
    value = 1.0 / (per_iter * iters)
    sample = (f"{steps} steps of {n} FP64 CG iterations (+1 refresh) of this 32^3x64 workload on the "
              f"{'reference' if kind == 'reference' else 'restated'} kernels, {threads} threads, {t:.1f} s; "
              f"solves/s = 1 / (seconds per iteration x {iters}), the iterations the reference's CG performed "
              f"in a full solve of this workload ({rec['seconds']} s on {rec['threads']} threads, true residual "
              f"{rec['true_resid_rel']:.2e}, oracle/workload_fp64_cg.json)")
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": warmup, "ms_per_step": t / steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": bench_config(ws),
            "extrapolation": {"measured": f"{steps * (n + 1)} iterations", "scaled_to": f"{iters} iterations"},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ GPU arm
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import cl2qcd_b200 as c2q
    from cl2qcd_b200 import build
    build.build()

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if args.serve:
        if rank == 0:
            rates = [float(x) for x in args.serve_rates.split(",")]
            for slots in [int(x) for x in args.serve_slots.split(",")]:
                for max_heavy in sorted({1, slots}):
                    res = serving_run(c2q, rates, args.serve_requests, slots=slots, max_heavy=max_heavy,
                                      log=lambda e: print(json.dumps({"serving_rate": e}), flush=True))
                    print(json.dumps({"metric": METRIC, "serving": res}), flush=True)
        return 0
    if args.phase == "mrhs":
        if rank == 0:
            print(json.dumps({"phase": "mrhs", "mrhs": mrhs_phase(c2q, args)}))
        return 0
    from cl2qcd_b200.replicas import Replicas
    replicas = Replicas("nccl", timeout_s=600, device=torch.device("cuda", local))

    def barrier():
        replicas.barrier()
        torch.cuda.synchronize()

    # a dedicated (non-default) stream: the library launches on it and the
    # torch events below record on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    system = c2q.System(local, stream.cuda_stream)
    lib = system.lib
    lat, g, b = inputs()
    gf = c2q.Gaugefield(system, lat, g)
    B = c2q.Spinorfield_eo(system, lat, b)
    X = c2q.Spinorfield_eo(system, lat)
    add = c2q.AdditionalParameters(KAPPA, mbar())
    A = c2q.host.QplusQminus_eo()
    P_mixed = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=40000, precision=args.precision,
                                   use_rec12=True)
    P_fp64 = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=40000, precision=64)

    def solve(P, rep=None):
        X.zero()
        c2q.host.cg(X, A, gf, B, P, add, rep)

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.phase == "large":
        out = large_volume(c2q, system, e0, e1)
        if rank == 0:
            print(json.dumps({"phase": "large", "large_volume": out}))
        system.close()
        return 0
    if args.phase == "dslash":
        out = dslash_gbs(c2q, system, lat, gf, b, e0, e1)
        if rank == 0:
            print(json.dumps({"phase": "dslash", "dslash_gbs": out}))
        system.close()
        return 0
    if args.phase == "mixed":
        for _ in range(args.warmup):
            solve(P_mixed)
        barrier()
        e0.record()
        for _ in range(args.steps):
            solve(P_mixed)
        e1.record()
        barrier()
        if rank == 0:
            print(json.dumps({"phase": "mixed", "ms_per_step": e0.elapsed_time(e1) / args.steps}))
        system.close()
        return 0

    # ---- FP64 reference solve on the GPU (reported beside the headline)
    rep64 = {}
    solve(P_fp64, rep64)
    x64 = X.dump()
    # the iteration count the reference's own CG needs for this target: its stop test
    # |r|^2 < prec (absolute, checked every 10 iterations) with prec = 1e-20 |b|^2
    b2 = float(np.vdot(b.reshape(-1), b.reshape(-1)))
    rep_ref_sem = {}
    solve(c2q.SolverParameters(solver="cg", prec=REL_TOL ** 2 * b2, cgmax=40000, precision=64), rep_ref_sem)
    ref_iters = rep_ref_sem["iterations"] + 1  # the reference returns the index of its last iteration
    barrier()
    e0.record()
    solve(P_fp64)
    e1.record()
    torch.cuda.synchronize()
    fp64_s = e0.elapsed_time(e1) / 1e3

    # ---- headline: mixed precision
    for _ in range(args.warmup):
        solve(P_mixed)
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = system.launch_count
    e0.record()
    reps = []
    for _ in range(args.steps):
        r = {}
        solve(P_mixed, r)
        reps.append(r)
    e1.record()
    barrier()
    launches = system.launch_count - launches0
    clk = clocks.stop()
    t = replicas.max_over_ranks(e0.elapsed_time(e1) / 1e3)
    xm = X.dump()
    err_vs_fp64 = float(np.linalg.norm(xm - x64) / np.linalg.norm(x64))
    value = ws * args.steps / t

    # ---- e2e through the public API with pinned host buffers
    src_host = torch.from_numpy(b.reshape(-1).copy()).pin_memory()
    sol_host = torch.empty(lat.seo * 24, dtype=torch.float64).pin_memory()
    src_np, sol_np = src_host.numpy(), sol_host.numpy()
    barrier()
    e0.record()
    for _ in range(args.steps):
        B.load(src_np)
        X.zero()
        c2q.host.cg(X, A, gf, B, P_mixed, add)
        lib.c2q_spinor_eo_download(X.h, sol_np)
    e1.record()
    barrier()
    te_seq = replicas.max_over_ranks(e0.elapsed_time(e1) / 1e3)
    x_seq = sol_np.copy()
    B.load(b)
    # the same with the transfers off the solve's path: two source and two solution
    # fields, and a copy stream (ordered by events against the context's stream)
    # that uploads the next step's source and downloads the previous step's
    # solution while the current solve runs
    copy = torch.cuda.Stream()
    cs = C.c_void_p(copy.cuda_stream)
    Bd = [c2q.Spinorfield_eo(system, lat) for _ in range(2)]
    Xd = [c2q.Spinorfield_eo(system, lat) for _ in range(2)]
    srcs = [torch.from_numpy(b.reshape(-1).copy()).pin_memory() for _ in range(2)]
    sols = [torch.empty(lat.seo * 24, dtype=torch.float64).pin_memory() for _ in range(2)]
    ev_up = [torch.cuda.Event() for _ in range(2)]
    ev_solved = [torch.cuda.Event() for _ in range(2)]
    ev_down = [torch.cuda.Event() for _ in range(2)]

    def xfer(fn, f, buf):
        if fn(f.h, buf.numpy(), cs) != 0:
            raise RuntimeError((lib.c2q_last_error(system.h) or b"").decode())

    barrier()
    e0.record()
    copy.wait_stream(stream)
    xfer(lib.c2q_spinor_eo_upload_async, Bd[0], srcs[0])
    ev_up[0].record(copy)
    for k in range(args.steps):
        cur, nxt = k % 2, (k + 1) % 2
        stream.wait_event(ev_up[cur])  # this step's source is on the device
        if k + 1 < args.steps:  # the next step's source (its field's last reader has finished)
            xfer(lib.c2q_spinor_eo_upload_async, Bd[nxt], srcs[nxt])
            ev_up[nxt].record(copy)
        if k >= 2:
            stream.wait_event(ev_down[cur])  # this solution field's previous download is done
        Xd[cur].zero()
        c2q.host.cg(Xd[cur], A, gf, Bd[cur], P_mixed, add)
        ev_solved[cur].record(stream)
        copy.wait_event(ev_solved[cur])
        xfer(lib.c2q_spinor_eo_download_async, Xd[cur], sols[cur])
        ev_down[cur].record(copy)
    stream.wait_stream(copy)
    e1.record()
    barrier()
    te = replicas.max_over_ranks(e0.elapsed_time(e1) / 1e3)
    e2e_diff = max(float(np.abs(sols[k % 2].numpy() - x_seq).max()) for k in range(min(2, args.steps)))

    # ---- roofline of the dominant kernel: the inner-precision dslash sweep, timed
    # per launch with CUDA events inside one more solve
    lib.c2q_ctx_profile(system.h, 1)
    rprof = {}
    solve(P_mixed, rprof)
    nl, ms, by = C.c_longlong(), C.c_double(), C.c_double()
    lib.c2q_ctx_profile_read(system.h, args.precision, C.byref(nl), C.byref(ms), C.byref(by))
    lib.c2q_ctx_profile(system.h, 0)
    peak, peak_kind = load_peaks()
    avg_s = ms.value / 1e3 / max(nl.value, 1)
    bytes_per_launch = by.value / max(nl.value, 1)
    achieved = bytes_per_launch / avg_s / 1e9 if avg_s > 0 else 0.0
    traffic = None
    tr = load_traffic()
    if tr and str(args.precision) in tr.get("dram_bytes_per_launch", {}):
        traffic = tr["dram_bytes_per_launch"][str(args.precision)]

    dg = dslash_gbs(c2q, system, lat, gf, b, e0, e1)

    # ---- FP32-inner variant of the mixed solver, same problem (reported beside)
    P32 = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=40000, precision=32, use_rec12=True)
    solve(P32)
    rep32 = {}
    e0.record()
    nrep = 5
    for _ in range(nrep):
        solve(P32, rep32)
    e1.record()
    torch.cuda.synchronize()
    fp32_s = e0.elapsed_time(e1) / 1e3 / nrep

    # ---- BiCGStab on Aee (the reference's default inversion solver), same gauge
    # field and source at kappa 0.12 (below the free critical kappa 1/8: at kappa
    # 0.16 the non-Hermitian Aee of these near-unit links has eigenvalues around
    # the origin and BiCGStab does not converge): FP64
    # against mixed precision (FP32 / FP16 inner, FP64 reliable updates), each to
    # the true residual 1e-10, timed over five solves after one untimed
    def bicgstab_section():
        kap = 0.12
        add_b = c2q.AdditionalParameters(kap, 2 * kap * MU)
        out = {"operator": "Aee", "variant": "bicgstab (fast)", "kappa": kap, "mu": MU}
        A_ee = c2q.host.Aee()
        for prec in (64, 32, 16):
            key = f"fp{prec}" if prec == 64 else f"mixed_fp{prec}"
            P_ = c2q.SolverParameters(solver="bicgstab", prec=0.0, rel_tol=REL_TOL, cgmax=3000, precision=prec,
                                      use_rec12=True)
            nrep_b = 5
            try:
                X.zero()
                c2q.host.bicgstab(X, A_ee, gf, B, P_, add_b, {})
                rep = {}
                e0.record()
                for _ in range(nrep_b):
                    X.zero()
                    c2q.host.bicgstab(X, A_ee, gf, B, P_, add_b, rep)
                e1.record()
                torch.cuda.synchronize()
            except Exception as e:  # reported, not fatal
                out[key] = {"error": repr(e)}
                continue
            sec = e0.elapsed_time(e1) / 1e3 / nrep_b
            out[key] = {"solves_per_s": 1.0 / sec, "iterations": rep["iterations"],
                        "reliable_updates": rep["reliable_updates"], "true_resid_rel": rep["true_resid_rel"]}
        if "solves_per_s" in out.get("mixed_fp16", {}) and "solves_per_s" in out.get("fp64", {}):
            out["speedup_mixed_fp16_vs_fp64"] = out["mixed_fp16"]["solves_per_s"] / out["fp64"]["solves_per_s"]
        return out

    bicg = bicgstab_section()

    # ---- batched multi-RHS: 12 spin-colour point sources at the origin, solved
    # together in batches of N = 1, 4, 8, 12 (mixed FP32 / FP16 inner, graph-
    # captured iterations), against the plain FP64 single-RHS solver on the same
    # sources
    def mrhs_section():
        srcs = [c2q.host.point_source(lat.seo, k) for k in range(12)]
        Bs = [c2q.Spinorfield_eo(system, lat, s_) for s_ in srcs]
        Xs = [c2q.Spinorfield_eo(system, lat) for _ in srcs]
        out = {"sources": "12 spin-colour point sources at the origin (spin k%4, colour k//4)",
               "operator": "QplusQminus_eo, same field and parameters", "graphs": True}
        reps64 = []
        for x_ in Xs:
            x_.zero()
        torch.cuda.synchronize()
        e0.record()
        for k in range(12):
            r = {}
            c2q.host.cg(Xs[k], A, gf, Bs[k], P_fp64, add, r)
            reps64.append(r)
        e1.record()
        torch.cuda.synchronize()
        t64 = e0.elapsed_time(e1) / 1e3
        out["fp64_single_rhs"] = {"solves_per_s": 12 / t64, "iterations": [r["iterations"] for r in reps64],
                                  "true_resid_rel_max": max(r["true_resid_rel"] for r in reps64)}
        # (the inner sweeps run in the temporal gauge by default; the last variant
        # keeps the plain gauge, for comparison)
        for prec, rec12, tg, sizes in ((32, True, True, (1, 4, 8, 12)), (16, True, True, (1, 4, 8, 12)),
                                       (16, False, True, (1, 4, 8, 12)), (16, True, False, (1, 12))):
            Pm = c2q.SolverParameters(solver="cg", prec=0.0, rel_tol=REL_TOL, cgmax=40000, precision=prec,
                                      use_rec12=rec12, use_graph=True, temporal_gauge=tg)
            res = {}
            for n in sizes:
                for x_ in Xs[:n]:
                    x_.zero()
                c2q.host.cg_multi(Xs[:n], A, gf, Bs[:n], Pm, add)  # warm-up: tuning, graph capture
                best = None
                for _rep in range(2):
                    for x_ in Xs[:n]:
                        x_.zero()
                    reps_ = []
                    torch.cuda.synchronize()
                    e0.record()
                    c2q.host.cg_multi(Xs[:n], A, gf, Bs[:n], Pm, add, reps_)
                    e1.record()
                    torch.cuda.synchronize()
                    tb = e0.elapsed_time(e1) / 1e3
                    if best is None or tb < best[0]:
                        best = (tb, reps_)
                tb, reps_ = best
                res[str(n)] = {"solves_per_s": n / tb, "seconds": tb,
                               "iterations": [r["iterations"] for r in reps_],
                               "reliable_updates": [r["reliable_updates"] for r in reps_],
                               "true_resid_rel_max": max(r["true_resid_rel"] for r in reps_),
                               "speedup_vs_fp64_single_rhs": (n / tb) / (12 / t64)}
            out[f"fp{prec}_inner" + ("" if rec12 else "_18real_links") + ("" if tg else "_plain_gauge")] = res
        return out

    mrhs = mrhs_section()
    config1 = config1_gpu(c2q, system, e0, e1)
    # serving stream at one arrival rate (the full sweep: --serve)
    serving = serving_run(c2q, [1.0], args.serve_requests) if rank == 0 and ws == 1 else None
    # config 5, 64^3x128 (BiCGStab bounded at 300 iterations: it does not converge there)
    large = None
    if rank == 0 and ws == 1 and not args.no_large:
        try:
            large = large_volume(c2q, system, e0, e1, bicgstab_cgmax=300,
                                 oracle_check_solution=not args.no_cpu_baseline)
        except Exception as e:  # reported, not fatal
            large = {"error": repr(e)}

    cpu_baseline = None
    rec_iters, _rec = recorded_fp64_iterations()
    check = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            check = oracle_check(g, b, xm, args.precision)
        except Exception as e:  # reported, never required
            check = {"error": repr(e)}
        try:
            cpu_baseline = cpu_reference_sample(g, b, rec_iters or ref_iters)
            cpu_baseline.pop("seconds_per_iteration", None)
            cpu_baseline.update(cpu_reference_extras(g, b))
        except Exception as e:  # the baseline is reported, never required
            cpu_baseline = {"value": None, "unit": "solves/s", "cores": os.cpu_count(), "kind": "reference",
                            "sample": f"unavailable: {e}"}

    if rank == 0:
        it_m = [r["iterations"] for r in reps]
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {16: "f16-fixed-point storage, f32 arithmetic, f64 reliable updates",
                      32: "f32 inner, f64 reliable updates", 64: "f64"}[args.precision],
            "data": "synthetic: seeded U=exp(i*0.25*H) gauge field (reunitarised in f64), gaussian source",
            "config": bench_config(ws, args.precision),
            "e2e": {"value": ws * args.steps / te, "unit": "solves/s", "h2d_bytes_per_step": lat.seo * 24 * 8,
                    "d2h_bytes_per_step": lat.seo * 24 * 8,
                    "mode": "public API, pinned host buffers; every step uploads its source and downloads its "
                            "solution, on a copy stream that overlaps the neighbouring steps' solves",
                    "max_abs_diff_vs_sequential": e2e_diff,
                    "sequential": {"value": ws * args.steps / te_seq,
                                   "mode": "upload, solve, download one after the other on one stream"}},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": f"{'dslash' if args.precision == 64 else 'pdslash'}_kernel<{args.precision}, 6, *>"
                                   " (all sweeps of one solve)",
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback 6.65 TB/s", "launches_timed": nl.value,
                         "bytes_per_launch": bytes_per_launch, "avg_launch_us": avg_s * 1e6},
            "cpu_baseline": cpu_baseline,
            "gpu_launches": launches,
            "clocks": clk,
            "mixed": {"iterations": it_m, "reliable_updates": [r["reliable_updates"] for r in reps],
                      "true_resid_rel": max(r["true_resid_rel"] for r in reps),
                      "rel_err_vs_fp64_solution": err_vs_fp64},
            "oracle_check": check,
            "fp64": {"solves_per_s": 1.0 / fp64_s, "iterations": rep64["iterations"],
                     "iterations_reference_semantics": ref_iters,
                     "iterations_reference_cg_on_cpu": rec_iters,
                     "true_resid_rel": rep64["true_resid_rel"], "seconds": fp64_s},
            "fp32_inner": {"solves_per_s": 1.0 / fp32_s, "iterations": rep32["iterations"],
                           "reliable_updates": rep32["reliable_updates"], "true_resid_rel": rep32["true_resid_rel"]},
            "speedup_mixed_vs_fp64": value / ws * fp64_s,
            "bicgstab": bicg,
            "dslash_gbs": dg,
            "multi_rhs": mrhs,
            "config1": config1,
            "serving": serving,
            "large_volume": large,
            "autotune": system.tune_report().strip().splitlines(),
        }
        print(json.dumps(line))
    system.close()
    replicas.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
