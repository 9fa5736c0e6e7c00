"""CPU: the oracle's input generators are bit-identical to the library's, so
that the CPU reference path can build the workload without loading the
library; the reference arm of bench.py loads only the oracle; the recorded
FP64 iteration count belongs to the benchmark workload."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("kind", ["port", "reference"])
@pytest.mark.parametrize("ns,nt,eps,seed", [(4, 4, 0.3, 1), (6, 8, 0.35, 99), (8, 8, 0.25, 20250)])
def test_gauge_generators_bit_identical(O, lib, kind, ns, nt, eps, seed):
    import cl2qcd_b200 as c2q
    if not O.available(kind):
        pytest.skip(f"oracle build {kind} absent")
    o = O.Oracle(kind)
    a = c2q.host.generate_gaugefield(c2q.Lattice(ns, nt, 1.0, 0.0), eps, seed)
    assert np.array_equal(a, o.gauge_generate(ns, nt, eps, seed))


@pytest.mark.parametrize("src", ["z2", "gaussian"])
def test_source_generators_bit_identical(port, lib, src):
    import cl2qcd_b200 as c2q
    for seed in (2, 777, 1 << 40):
        assert np.array_equal(c2q.host.generate_source(4099, src, seed), port.source_generate(4099, src, seed))


def test_recorded_workload_matches_bench():
    sys.path.insert(0, ROOT)
    import bench
    iters, rec = bench.recorded_fp64_iterations()
    assert iters == rec["cg_returned"] + 1 and iters > 0
    assert rec["true_resid_rel"] <= 1e-10
    assert rec["oracle"] in ("reference", "port")


def test_reference_arm_loads_only_the_oracle():
    """bench.py --impl reference: the reference's kernels on the host, the
    library never mapped, and the same `config` as the GPU arm's."""
    code = (
        "import sys, json\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0']\n"
        "import bench\n"
        "bench.run_reference(bench.parse(), budget_s=1.0)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'lib_mapped': 'libc2q_b200' in maps, 'torch': 'torch' in sys.modules,\n"
        "                  'config': bench.bench_config(1)}))\n"
    )
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
    line, probe = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"] == probe["config"]
    assert not probe["lib_mapped"] and not probe["torch"]
