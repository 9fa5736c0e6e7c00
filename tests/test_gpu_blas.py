"""GPU parity of the eo BLAS, reductions, tm site-diagonal ops and layout conversions."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(port, system):
    import cl2qcd_b200 as c2q
    port.set_lattice(8, 4)
    L = c2q.Lattice(8, 4)
    x = port.pseudo_randomize(port.seo, 1) - 0.5
    y = port.pseudo_randomize(port.seo, 2) - 0.5
    z = port.pseudo_randomize(port.seo, 3) - 0.5
    X, Y, Z = (c2q.Spinorfield_eo(system, L, a) for a in (x, y, z))
    return c2q, L, x, y, z, X, Y, Z


def test_upload_download_roundtrip(env):
    c2q, L, x, y, z, X, Y, Z = env
    assert np.array_equal(X.dump(), x)


def test_saxpy_family(env, port, system):
    c2q, L, x, y, z, X, Y, Z = env
    O = c2q.Spinorfield_eo(system, L)
    a, b = 0.37 - 1.2j, -0.8 + 0.25j
    c2q.host.saxpy(O, a, X, Y)
    assert rel_l2(O.dump(), port.saxpy(a, x, y)) < 1e-15
    c2q.host.saxpy_AND_gamma5_eo(O, a, X, Y)
    assert rel_l2(O.dump(), port.saxpy_gamma5(a, x, y)) < 1e-15
    c2q.host.sax(O, a, X)
    assert rel_l2(O.dump(), port.sax(a, x)) < 1e-15
    c2q.host.saxsbypz(O, a, X, b, Y, Z)
    assert rel_l2(O.dump(), port.saxsbypz(a, x, b, y, z)) < 1e-15
    c2q.host.copyData(O, Z)
    assert np.array_equal(O.dump(), z)
    n = c2q.host.saxpy_AND_squarenorm(O, a, X, Y)
    ref_out, ref_n = port.saxpy_squarenorm(a, x, y)
    assert rel_l2(O.dump(), ref_out) < 1e-15 and n == pytest.approx(ref_n, rel=1e-13)


def test_reductions(env, port):
    c2q, L, x, y, z, X, Y, Z = env
    sp = c2q.host.scalar_product(X, Y)
    ref = port.scalar_product(x, y)
    assert abs(sp - ref) <= 1e-13 * abs(ref)
    assert c2q.host.squarenorm(X) == pytest.approx(port.squarenorm(x), rel=1e-13)
    # deterministic: the same inputs give bitwise the same reduction
    assert all(c2q.host.scalar_product(X, Y) == sp for _ in range(5))


def test_gamma5_and_diag(env, port, system, O):
    c2q, L, x, y, z, X, Y, Z = env
    W = c2q.Spinorfield_eo(system, L, x)
    W.gamma5()
    assert np.array_equal(W.dump(), port.gamma5_eo(x))
    mubar = 0.0123
    for name, which in [("M_tm_sitediagonal", O.DIAG_M), ("M_tm_inverse_sitediagonal", O.DIAG_MINV),
                        ("M_tm_sitediagonal_minus", O.DIAG_M_MINUS),
                        ("M_tm_inverse_sitediagonal_minus", O.DIAG_MINV_MINUS),
                        ("M_tm_sitediagonal_AND_gamma5_eo", O.DIAG_M_G5),
                        ("M_tm_sitediagonal_minus_AND_gamma5_eo", O.DIAG_M_MINUS_G5)]:
        getattr(c2q.host, name)(W, X, mubar)
        assert rel_l2(W.dump(), port.tm_diag(x, mubar, which)) < 1e-15, name


def test_cold_zero_and_convert(env, port, system):
    c2q, L, x, y, z, X, Y, Z = env
    W = c2q.Spinorfield_eo(system, L)
    W.cold()
    assert rel_l2(W.dump(), port.cold_eo()) < 1e-16
    W.zero()
    assert not W.dump().any()
    full = port.pseudo_randomize(port.vol, 8)
    E, Od = c2q.Spinorfield_eo(system, L), c2q.Spinorfield_eo(system, L)
    c2q.host.convert_to_eoprec(E, Od, full)
    e_ref, o_ref = port.convert_to_eo(full)
    assert np.array_equal(E.dump(), e_ref) and np.array_equal(Od.dump(), o_ref)
    assert np.array_equal(c2q.host.convert_from_eoprec(E, Od), full)


def test_bad_arguments_raise(env, system):
    c2q, L, x, y, z, X, Y, Z = env
    other = c2q.Spinorfield_eo(system, c2q.Lattice(4, 4))
    with pytest.raises(c2q.host.InvalidParameters):
        c2q.host.saxpy(other, 1.0, X, Y)
    with pytest.raises(c2q.host.InvalidParameters):
        c2q.Spinorfield_eo(system, c2q.Lattice(5, 4))


def test_async_transfers_round_trip(system, port):
    """c2q_spinor_eo_upload_async / download_async: enqueued without waiting, on the
    context's stream or on a copy stream of the caller's; the data arrive after
    that stream synchronises; FP32 fields are refused."""
    import torch
    import cl2qcd_b200 as c2q
    lib = system.lib
    L = c2q.Lattice(4, 8)
    port.set_lattice(4, 8)
    a = np.ascontiguousarray(port.pseudo_randomize(L.seo, 5))
    f = c2q.Spinorfield_eo(system, L)
    assert lib.c2q_spinor_eo_upload_async(f.h, a, None) == 0
    out = np.zeros_like(a)
    assert lib.c2q_spinor_eo_download_async(f.h, out, None) == 0
    system.synchronize()
    assert np.array_equal(out, a)
    copy = torch.cuda.Stream()
    b = np.ascontiguousarray(port.pseudo_randomize(L.seo, 6))
    assert lib.c2q_spinor_eo_upload_async(f.h, b, C.c_void_p(copy.cuda_stream)) == 0
    out2 = np.zeros_like(b)
    assert lib.c2q_spinor_eo_download_async(f.h, out2, C.c_void_p(copy.cuda_stream)) == 0
    copy.synchronize()
    assert np.array_equal(out2, b)
    g = c2q.Spinorfield_eo(system, L, a, precision=32)
    assert lib.c2q_spinor_eo_upload_async(g.h, a, None) != 0
    assert lib.c2q_spinor_eo_download_async(g.h, out, None) != 0
