"""GPU: the device-driven eo BiCGStab (fast and save variants of
physics/algorithms/solvers/bicgstab.cpp:401-733).  Its scalars live in device
memory, the host reads |r|^2 one iteration behind the queue, and a device halt
flag empties every launch queued behind the iteration that stops.

* The returned iterate is the reference loop's: a converged solve gives, bit for
  bit, the x of the same solve cut off by solverMaxIterations where the reference
  would have stopped -- nothing queued behind the stop touched x.
* Iteration counts and solutions agree with the oracle's restatement of the
  reference's BiCGStab for refresh intervals that put refreshes inside the solve,
  including one that makes the solve stop on the test that follows a refresh.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

KAPPA, MU = 0.13, 0.05
CODE = {"bicgstab": 2, "bicgstab_save": 3}


def _prob(port, c2q, system, ns=8, nt=4, seed=3):
    port.set_lattice(ns, nt, 1.0, 0.0)
    L = c2q.Lattice(ns, nt, 1.0, 0.0)
    g = c2q.host.generate_gaugefield(L, 0.3, seed)
    gf = c2q.Gaugefield(system, L, g)
    b = c2q.host.generate_source(port.seo, "z2", seed + 100)
    return L, g, gf, b


def _solve(c2q, system, L, gf, b, variant, cgmax, refresh=100, prec=1e-20):
    X, B = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L, b)
    rep = {}
    try:
        it = c2q.host.bicgstab(X, c2q.host.Aee(), gf, B,
                               c2q.SolverParameters(solver=variant, prec=prec, cgmax=cgmax, iter_refresh=refresh),
                               c2q.AdditionalParameters(KAPPA, 2 * KAPPA * MU), rep)
    except c2q.SolverDidNotSolve:
        it = None
    return it, X.dump(), rep


@pytest.mark.parametrize("variant", ["bicgstab", "bicgstab_save"])
def test_stop_leaves_the_reference_iterate(port, system, variant):
    """The fast variant returns j from the test at the top of iteration j, after
    iterations 0 .. j-1: the same x as a solve limited to j iterations.  The save
    variant returns j from the test at the end of iteration j: the same x as a
    solve limited to j + 1 iterations (which queues nothing behind it)."""
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system)
    j, x_conv, rep = _solve(c2q, system, L, gf, b, variant, 1000)
    assert j and j > 5, rep
    cut = j if variant == "bicgstab" else j + 1
    j_cut, x_cut, _ = _solve(c2q, system, L, gf, b, variant, cut)
    assert j_cut == (None if variant == "bicgstab" else j)
    assert np.array_equal(x_conv, x_cut)


@pytest.mark.parametrize("variant", ["bicgstab", "bicgstab_save"])
def test_refresh_intervals_match_oracle(port, system, O, variant):
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system)
    mubar = 2 * KAPPA * MU
    j, _, _ = _solve(c2q, system, L, gf, b, variant, 1000)
    # refreshes inside the solve; refresh = j puts a refresh on the stopping iteration
    for refresh in (10, 17, j):
        x_ref = np.zeros_like(b)
        it_ref = port.bicgstab(x_ref, O.OP_AEE, b, g, KAPPA, mubar,
                               params=O.SolverParams(prec=1e-20, cgmax=3000, iter_refresh=refresh,
                                                     solver=CODE[variant]))
        it, x, rep = _solve(c2q, system, L, gf, b, variant, 3000, refresh=refresh)
        assert it_ref > 0 and it is not None, (refresh, it_ref, rep)
        assert abs(it - it_ref) <= 2, (refresh, it, it_ref)
        assert rel_l2(x, x_ref) < 1e-8, refresh
        assert rep["true_resid_rel"] < 1e-9, rep


def test_dslash_applications_counted_once(port, system):
    """Sweeps skipped behind the stop are not reported: fast variant, no refresh
    after the first, stop at the top of iteration j: one refresh, two Aee per
    iteration, the final true residual; two sweeps per Aee."""
    import cl2qcd_b200 as c2q
    L, g, gf, b = _prob(port, c2q, system)
    j, _, rep = _solve(c2q, system, L, gf, b, "bicgstab", 1000)
    assert rep["dslash_applications"] == 2 * (1 + 2 * j + 1), (j, rep)


@pytest.mark.parametrize("variant", ["bicgstab", "bicgstab_save"])
@pytest.mark.parametrize("precision", [32, 16])
@pytest.mark.parametrize("shape", [(8, 4), (4, 8)])
def test_mixed_iterations_track_fp64(port, system, variant, precision, shape):
    """The inner BiCGStab on FP32 / FP16 fields (fused x / rn update with its two
    reductions, (rhat, v) reduced in the operator's last sweep) needs about the
    iterations of the FP64 solve, over its reliable updates, from a zero
    and from a cold start: an inner iteration that reduced stale or wrong values
    would still end in a converged outer solve, but only after many more."""
    import cl2qcd_b200 as c2q
    ns, nt = shape
    L, g, gf, b = _prob(port, c2q, system, ns, nt)
    add = c2q.AdditionalParameters(0.14, 2 * 0.14 * 0.05)
    its = {}
    for prec in (64, precision):
        for cold in (False, True):
            X, B = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L, b)
            if cold:
                system.lib.c2q_spinor_eo_cold(X.h)
            rep = {}
            c2q.host.bicgstab(X, c2q.host.Aee(), gf, B,
                              c2q.SolverParameters(solver=variant, prec=0.0, rel_tol=1e-11, cgmax=2000,
                                                   precision=prec), add, rep)
            assert rep["true_resid_rel"] <= 1e-11, rep
            its[prec, cold] = rep["iterations"]
    for cold in (False, True):
        assert its[precision, cold] <= 1.3 * its[64, cold] + 5, its
