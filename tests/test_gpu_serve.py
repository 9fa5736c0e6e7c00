"""GPU: the serving loop (c2q_server_*).

Requests that run together on the device (several slots, overlapping in
time) must give the same solutions as the same requests run alone, one after
the other (stated tolerance: 1e-12 relative; the arithmetic does not depend on
what else runs, so the results are expected to be identical); every solution
meets the true-residual bar 1e-10, checked against the oracle operator; the
HBM budget serialises requests that do not fit together; a request that can
never fit fails with C2Q_OOM without running.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REQS = [  # (lattice index, gauge id, kappa, mu, nsrc, seed)
    (0, 1, 0.150, 0.010, 3, 11),
    (1, 2, 0.145, 0.005, 2, 22),
    (0, 1, 0.155, 0.020, 1, 33),
    (1, 3, 0.140, 0.002, 4, 44),
    (0, 4, 0.160, 0.008, 2, 55),
    (1, 2, 0.152, 0.015, 3, 66),
]
LATS = [(8, 8), (8, 16)]


def _setup(c2q, server):
    lats = [c2q.Lattice(ns, nt, 1.0, 0.0) for ns, nt in LATS]
    gauges = {1: (0, 0.30, 101), 2: (1, 0.25, 102), 3: (1, 0.35, 103), 4: (0, 0.20, 104)}
    fields = {}
    for gid, (li, eps, seed) in gauges.items():
        g = c2q.host.generate_gaugefield(lats[li], eps, seed)
        server.add_gauge(gid, lats[li], g)
        fields[gid] = g
    return lats, fields


def _run(c2q, slots, budget=0):
    server = c2q.host.Server(0, slots=slots, hbm_budget=budget, precision=16)
    lats, fields = _setup(c2q, server)
    sols, tickets = [], []
    for (li, gid, kappa, mu, n, seed) in REQS:
        sol = np.zeros((n, lats[li].seo, 24))
        sols.append(sol)
        tickets.append(server.submit(lats[li], gid, kappa, mu, n, seed, solutions=sol))
    results = [server.wait(t) for t in tickets]
    server.close()
    return lats, fields, sols, results


def test_same_result_alone_and_in_the_mix(port, O):
    import cl2qcd_b200 as c2q
    lats, fields, mixed, rmix = _run(c2q, slots=3)
    # the same requests, one at a time
    server = c2q.host.Server(0, slots=1, precision=16)
    _setup(c2q, server)
    for i, (li, gid, kappa, mu, n, seed) in enumerate(REQS):
        sol = np.zeros((n, lats[li].seo, 24))
        r = server.wait(server.submit(lats[li], gid, kappa, mu, n, seed, solutions=sol))
        assert r["status"] == 0 and rmix[i]["status"] == 0, (r, rmix[i])
        assert r["iterations_max"] == rmix[i]["iterations_max"]
        d = np.max(np.abs(sol - mixed[i])) / np.max(np.abs(sol))
        assert d <= 1e-12, (i, d)
    server.close()
    # every solution against the oracle operator
    for i, (li, gid, kappa, mu, n, seed) in enumerate(REQS):
        assert rmix[i]["true_resid_rel_max"] <= 1e-10
        port.set_lattice(*LATS[li], 1.0, 0.0)
        for k in range(n):
            b = c2q.host.generate_source(lats[li].seo, "z2", seed + k)
            r = port.apply(O.OP_QPQM_EO, mixed[i][k], fields[gid], kappa, 2 * kappa * mu)
            assert np.linalg.norm(r - b) / np.linalg.norm(b) <= 1.5e-10, (i, k)


def test_requests_overlap_on_the_device():
    import cl2qcd_b200 as c2q
    _, _, _, res = _run(c2q, slots=3)
    spans = sorted((r["t_admit"], r["t_done"]) for r in res)
    overlapped = any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    assert overlapped, spans


def test_budget_serialises_requests():
    import cl2qcd_b200 as c2q
    probe = c2q.host.Server(0, slots=1)
    lats, _ = _setup(c2q, probe)
    gauge_bytes = probe.stats()["gauge_bytes"]
    probe.close()
    biggest = max(c2q.host.request_footprint(lats[li], n, 16) for (li, _, _, _, n, _) in REQS)
    # room for the largest request, never for two of them
    budget = gauge_bytes + int(1.5 * biggest)
    _, _, _, res = _run(c2q, slots=3, budget=budget)
    assert all(r["status"] == 0 for r in res), res
    spans = sorted((r["t_admit"], r["t_done"], r["footprint_bytes"]) for r in res)
    for i in range(len(spans) - 1):
        a, b = spans[i], spans[i + 1]
        if b[0] < a[1]:  # overlapping in time: they must fit together
            assert a[2] + b[2] <= 1.5 * biggest


def test_request_that_never_fits_fails_with_oom():
    import cl2qcd_b200 as c2q
    server = c2q.host.Server(0, slots=1, hbm_budget=1 << 26)  # 64 MB: the gauge field fits, 64 sources do not
    L = c2q.Lattice(8, 8, 1.0, 0.0)
    server.add_gauge(7, L, c2q.host.generate_gaugefield(L, 0.3, 7))
    r = server.wait(server.submit(L, 7, 0.15, 0.01, 64, 1))
    assert r["status"] == -4  # C2Q_OOM
    r = server.wait(server.submit(L, 8, 0.15, 0.01, 1, 1))  # unknown gauge id
    assert r["status"] == -5
    server.close()


def test_heavy_requests_run_one_at_a_time():
    """With every request counted as heavy (threshold 1 site-source) and at most
    one heavy request at a time, three slots run the requests one after another;
    with the limit lifted they overlap again."""
    import cl2qcd_b200 as c2q
    for max_heavy, expect_overlap in ((1, False), (3, True)):
        server = c2q.host.Server(0, slots=3, precision=16)
        server.set_heavy_limit(1, max_heavy)
        lats, _ = _setup(c2q, server)
        tickets = [server.submit(lats[li], gid, kappa, mu, n, seed) for (li, gid, kappa, mu, n, seed) in REQS]
        res = [server.wait(t) for t in tickets]
        server.close()
        assert all(r["status"] == 0 for r in res), res
        spans = sorted((r["t_admit"], r["t_done"]) for r in res)
        overlapped = any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
        assert overlapped == expect_overlap, (max_heavy, spans)
