"""CPU: the C-ABI library loads and exports exactly what include/*.h declares;
the host-side input generators (no GPU) behave."""
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names |= set(re.findall(r"C2Q_EXPORT\s+[\w\s\*]+?\b(c2q_\w+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"c2q_dslash_eo", "c2q_cg", "c2q_bicgstab", "c2q_perform_inversion_eo", "c2q_apply_eo"} <= names


def test_library_exports_every_declared_symbol(lib):
    import ctypes
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding knows the signature of each
    from cl2qcd_b200 import _lib
    assert declared_symbols() <= set(_lib.SIGNATURES), declared_symbols() - set(_lib.SIGNATURES)
    assert lib.c2q_version().startswith(b"cl2qcd-b200")


def test_no_device_is_reported_cleanly_or_context_works(lib):
    import ctypes
    h = ctypes.c_void_p()
    rc = lib.c2q_ctx_create(ctypes.byref(h), 0, None)
    if rc == 0:
        lib.c2q_ctx_destroy(h)
    else:
        assert rc == -7  # C2Q_NO_DEVICE on a machine without a GPU


def test_gauge_generator_su3(lib):
    import cl2qcd_b200 as c2q
    L = c2q.Lattice(4, 4)
    g = c2q.host.generate_gaugefield(L, 0.3, 7)
    U = (g[:, 0::2] + 1j * g[:, 1::2]).reshape(-1, 3, 3)
    eye = np.eye(3)
    assert np.abs(U @ U.conj().transpose(0, 2, 1) - eye).max() < 1e-14
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-14
    g2 = c2q.host.generate_gaugefield(L, 0.3, 7)
    assert np.array_equal(g, g2)  # deterministic, thread-count independent streams
    assert not np.array_equal(g, c2q.host.generate_gaugefield(L, 0.3, 8))
    # small eps -> close to the identity; the generator is exp(i eps H)
    gs = c2q.host.generate_gaugefield(L, 1e-6, 7)
    Us = (gs[:, 0::2] + 1j * gs[:, 1::2]).reshape(-1, 3, 3)
    assert np.abs(Us - eye).max() < 1e-4


def test_source_generators(lib):
    import cl2qcd_b200 as c2q
    z = c2q.host.generate_source(1000, "z2", 3)
    assert np.allclose(np.abs(z), 1 / np.sqrt(2))
    gs = c2q.host.generate_source(20000, "gaussian", 3)
    assert abs(gs.mean()) < 0.02 and abs(gs.std() - 1) < 0.02


def test_request_footprint_is_monotone():
    """The serving admission footprint (host arithmetic only) grows with the
    number of sources and the volume, and FP16 inner fields need less than FP32."""
    import cl2qcd_b200 as c2q
    small, big = c2q.Lattice(16, 32), c2q.Lattice(48, 96)
    f = c2q.host.request_footprint
    assert 0 < f(small, 1) < f(small, 2) < f(small, 12) < f(big, 1)
    assert f(big, 12, 16) < f(big, 12, 32) <= f(big, 12, 64)
    # 48^3x96 with 12 sources: about 53 GB, 32^3x64 with 12 about 10.5 GB
    assert 50e9 < f(big, 12, 16) < 56e9
    assert 10e9 < f(c2q.Lattice(32, 64), 12, 16) < 11e9
