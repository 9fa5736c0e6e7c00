"""GPU: the allocation-free scalar product (c2q_scalar_product_eo_noalloc).

It serves callers that cannot allocate device memory (a memory pool that owns
the GPU, loops that cannot take an allocation's synchronisation, host programs
that forbid plugins to allocate).  The caller owns every buffer; the library
uses a fixed scratch array of its own.  This test builds the caller-owned
buffers with torch, calls the entry point through the C ABI twice in a row
(different inputs, so a stale scratch would show), and compares each result
with the existing c2q_scalar_product on the same fields.  It sits in a file of
its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _soa(aos, stride):
    """Host AoS eo field (Seo, 24) -> the library's FP64 device layout (12 lanes of double2, lane stride `stride`)."""
    n = aos.shape[0]
    lanes = np.zeros((12, stride, 2))
    lanes[:, :n, :] = aos.reshape(n, 12, 2).transpose(1, 0, 2)
    return lanes


def test_noalloc_scalar_product_matches_existing(lib):
    torch = pytest.importorskip("torch")
    import cl2qcd_b200 as c2q

    torch.cuda.init()
    system = c2q.System(0)
    lat = c2q.Lattice(8, 8, 1.0, 0.0)  # 2048 eo sites
    n = lat.seo
    stride = (n + 63) // 64 * 64
    stream = torch.cuda.current_stream()
    rel_tol = 1e-13
    try:
        for call, seeds in enumerate([(11, 12), (21, 22)]):
            x = c2q.host.generate_source(n, "gaussian", seeds[0])
            y = c2q.host.generate_source(n, "gaussian", seeds[1])
            # existing entry point
            X, Y = c2q.Spinorfield_eo(system, lat, x), c2q.Spinorfield_eo(system, lat, y)
            expected = c2q.host.scalar_product(X, Y)
            # allocation-free entry point on caller-owned device buffers
            xd = torch.from_numpy(_soa(x, stride)).cuda()
            yd = torch.from_numpy(_soa(y, stride)).cuda()
            res = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
            rc = lib.c2q_scalar_product_eo_noalloc(C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), n, stride,
                                                   C.c_void_p(res.data_ptr()), C.c_void_p(stream.cuda_stream))
            assert rc == 0, f"call {call}: status {rc}"
            torch.cuda.synchronize()
            got = complex(res[0].item(), res[1].item())
            assert abs(got - expected) <= rel_tol * abs(expected), (call, got, expected)
            # and against numpy directly
            ref = np.vdot(x[:, 0::2] + 1j * x[:, 1::2], y[:, 0::2] + 1j * y[:, 1::2])
            assert abs(got - ref) <= 1e-12 * abs(ref)
            del X, Y
    finally:
        system.close()


def test_noalloc_rejects_oversized_fields(lib):
    torch = pytest.importorskip("torch")
    n = 4194304 + 1  # C2Q_NOALLOC_MAX_SITES + 1
    dummy = torch.zeros(2, dtype=torch.float64, device="cuda")
    p = C.c_void_p(dummy.data_ptr())
    assert lib.c2q_scalar_product_eo_noalloc(p, p, n, n, p, None) == -5  # C2Q_BAD_ARG, nothing launched
    # misaligned caller buffers (a view at an odd offset) are refused before any launch
    base = dummy.data_ptr()
    assert lib.c2q_scalar_product_eo_noalloc(C.c_void_p(base + 8), p, 64, 64, p, None) == -5
    assert lib.c2q_scalar_product_eo_noalloc(p, C.c_void_p(base + 8), 64, 64, p, None) == -5
    assert lib.c2q_scalar_product_eo_noalloc(p, p, 64, 64, C.c_void_p(base + 4), None) == -5
