"""CPU oracle for the tm-Wilson eo hot path -- TEST INFRASTRUCTURE ONLY.

Two builds of the same C API (``c2qo_*``) live under ``oracle/_ref/``:

* ``libc2q_oracle.so`` -- this project's own C restatement of the reference
  kernels (``oracle_kernels_port.c``) plus the restated control flow of
  ``physics/fermionmatrix/fermionmatrix.cpp``, ``physics/algorithms/solvers/cg.cpp``,
  ``bicgstab.cpp`` and ``physics/algorithms/inversion.cpp`` ("port");
* ``libc2q_ref.so`` -- the same control flow on the reference's own OpenCL-C
  kernels compiled as C ("reference").

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package; the product never does.

All fields are numpy float64 arrays in the reference's host formats: eo spinor
fields ``(Seo, 24)``, full fields ``(V, 24)``, gauge fields ``(4*V, 18)`` at link
``mu + 4*site``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_REF_DIR = os.path.join(_HERE, "_ref")

WILSON, TWISTEDMASS = 0, 1
OP_AEE, OP_AEE_MINUS, OP_QPLUS_EO, OP_QMINUS_EO, OP_QPQM_EO, OP_AEE_G5, OP_AEE_MINUS_G5 = range(7)
DIAG_M, DIAG_MINV, DIAG_M_MINUS, DIAG_MINV_MINUS, DIAG_M_G5, DIAG_M_MINUS_G5 = range(6)
EVEN, ODD = 0, 1
SOLVER_STUCK, DID_NOT_SOLVE = -1, -2


class SolverParams(C.Structure):
    """Mirror of ``c2qo_solver_params`` (reference defaults, meta/parametersSolver.cpp:74-107)."""

    _fields_ = [
        ("prec", C.c_double),
        ("cgmax", C.c_int),
        ("iter_refresh", C.c_int),
        ("resid_check_every", C.c_int),
        ("min_iter", C.c_int),
        ("merge_spinor", C.c_int),
        ("merge_fermion", C.c_int),
        ("solver", C.c_int),
    ]

    def __init__(self, prec=1e-23, cgmax=1000, iter_refresh=100, resid_check_every=10, min_iter=0,
                 merge_spinor=0, merge_fermion=0, solver=2):
        super().__init__(prec, cgmax, iter_refresh, resid_check_every, min_iter, merge_spinor, merge_fermion,
                         solver)


_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Compile the oracle libraries with ``make`` (outputs under oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all" if ref else "_ref/libc2q_oracle.so"], check=True)


class Oracle:
    """ctypes view of one oracle build (``kind`` = "port" or "reference")."""

    def __init__(self, kind: str = "port"):
        name = {"port": "libc2q_oracle.so", "reference": "libc2q_ref.so"}[kind]
        path = os.path.join(_REF_DIR, name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library {path} is not built (run make -C oracle)")
        self.kind = kind
        L = self.lib = C.CDLL(path)
        i, d, sz = C.c_int, C.c_double, C.c_size_t
        sig = {
            "c2qo_backend": (C.c_char_p, []),
            "c2qo_set_lattice": (None, [i, i, d, d, i, d, i, d]),
            "c2qo_dslash_eo": (None, [_D, _D, _D, i, d]),
            "c2qo_dslash_tm_inv_eo": (None, [_D, _D, _D, i, d, d, i]),
            "c2qo_tm_diag": (None, [_D, _D, d, i]),
            "c2qo_gamma5_eo": (None, [_D]),
            "c2qo_saxpy": (None, [_D, d, d, _D, _D]),
            "c2qo_saxpy_gamma5": (None, [_D, d, d, _D, _D]),
            "c2qo_sax": (None, [_D, d, d, _D]),
            "c2qo_saxsbypz": (None, [_D, d, d, _D, d, d, _D, _D]),
            "c2qo_scalar_product": (None, [_D, _D, C.POINTER(d), C.POINTER(d)]),
            "c2qo_squarenorm": (d, [_D]),
            "c2qo_squarenorm_full": (d, [_D]),
            "c2qo_saxpy_squarenorm": (d, [_D, d, d, _D, _D]),
            "c2qo_cold": (None, [_D]),
            "c2qo_zero": (None, [_D]),
            "c2qo_convert_to_eo": (None, [_D, _D, _D]),
            "c2qo_convert_from_eo": (None, [_D, _D, _D]),
            "c2qo_m_tm_plus": (None, [_D, _D, _D, d, d]),
            "c2qo_m_tm_minus": (None, [_D, _D, _D, d, d]),
            "c2qo_gamma5_full": (None, [_D]),
            "c2qo_apply": (None, [i, _D, _D, _D, d, d, i, i]),
            "c2qo_cg": (i, [_D, i, _D, _D, d, d, i, C.POINTER(SolverParams)]),
            "c2qo_bicgstab": (i, [_D, i, _D, _D, d, d, i, C.POINTER(SolverParams)]),
            "c2qo_perform_inversion_eo": (i, [_D, _D, _D, d, d, i, C.POINTER(SolverParams), C.POINTER(i)]),
            "c2qo_fermion_force_eo": (None, [_D, _D, _D, _D, i, d]),
            "c2qo_gm_squarenorm": (d, [_D]),
            "c2qo_fermion_force_full": (None, [_D, _D, _D, _D, d]),
            "c2qo_calc_fermion_force_eo": (i, [_D, _D, _D, d, d, i, C.POINTER(SolverParams)]),
            "c2qo_calc_s_fermion_eo": (d, [_D, _D, d, d, i, C.POINTER(SolverParams), C.POINTER(i)]),
            "c2qo_pseudo_randomize": (None, [_D, sz, i]),
            "c2qo_fill_gauge": (None, [_D, sz, i]),
            "c2qo_fill_ascending_complex": (None, [_D, sz]),
            "c2qo_count_sf": (d, [_D, sz]),
            "c2qo_gauge_generate": (i, [_D, i, i, d, C.c_ulonglong]),
            "c2qo_source_generate": (i, [_D, sz, i, C.c_ulonglong]),
        }
        for fn, (res, args) in sig.items():
            f = getattr(L, fn)
            f.restype = res
            f.argtypes = args
        self.ns = self.nt = None

    # ---- lattice ----
    def set_lattice(self, ns, nt, theta_t=0.0, theta_s=0.0, cp_re=None, cp_im=None):
        self.ns, self.nt = ns, nt
        self.lib.c2qo_set_lattice(ns, nt, theta_t, theta_s, int(cp_re is not None), cp_re or 0.0,
                                  int(cp_im is not None), cp_im or 0.0)

    @property
    def vol(self):
        return self.ns ** 3 * self.nt

    @property
    def seo(self):
        return self.vol // 2

    def eo_field(self):
        return np.zeros((self.seo, 24))

    def full_field(self):
        return np.zeros((self.vol, 24))

    # ---- kernels ----
    def dslash_eo(self, inp, gauge, evenodd, kappa):
        out = self.eo_field()
        self.lib.c2qo_dslash_eo(out, inp, gauge, evenodd, kappa)
        return out

    def dslash_tm_inv_eo(self, inp, gauge, evenodd, kappa, mubar, minus=False):
        out = self.eo_field()
        self.lib.c2qo_dslash_tm_inv_eo(out, inp, gauge, evenodd, kappa, mubar, int(minus))
        return out

    def tm_diag(self, inp, mubar, which):
        out = self.eo_field()
        self.lib.c2qo_tm_diag(out, inp, mubar, which)
        return out

    def gamma5_eo(self, inp):
        out = np.array(inp, copy=True)
        self.lib.c2qo_gamma5_eo(out)
        return out

    def saxpy(self, alpha, x, y):
        out = self.eo_field()
        self.lib.c2qo_saxpy(out, alpha.real, alpha.imag, x, y)
        return out

    def saxpy_gamma5(self, alpha, x, y):
        out = self.eo_field()
        self.lib.c2qo_saxpy_gamma5(out, alpha.real, alpha.imag, x, y)
        return out

    def sax(self, alpha, x):
        out = self.eo_field()
        self.lib.c2qo_sax(out, alpha.real, alpha.imag, x)
        return out

    def saxsbypz(self, alpha, x, beta, y, z):
        out = self.eo_field()
        self.lib.c2qo_saxsbypz(out, alpha.real, alpha.imag, x, beta.real, beta.imag, y, z)
        return out

    def scalar_product(self, x, y):
        re, im = C.c_double(), C.c_double()
        self.lib.c2qo_scalar_product(x, y, C.byref(re), C.byref(im))
        return complex(re.value, im.value)

    def squarenorm(self, x):
        return self.lib.c2qo_squarenorm(x)

    def squarenorm_full(self, x):
        return self.lib.c2qo_squarenorm_full(x)

    def saxpy_squarenorm(self, alpha, x, y):
        out = self.eo_field()
        n = self.lib.c2qo_saxpy_squarenorm(out, alpha.real, alpha.imag, x, y)
        return out, n

    def cold_eo(self):
        out = self.eo_field()
        self.lib.c2qo_cold(out)
        return out

    def convert_to_eo(self, full):
        even, odd = self.eo_field(), self.eo_field()
        self.lib.c2qo_convert_to_eo(even, odd, full)
        return even, odd

    def convert_from_eo(self, even, odd):
        full = self.full_field()
        self.lib.c2qo_convert_from_eo(full, even, odd)
        return full

    def m_tm_plus(self, inp, gauge, kappa, mubar):
        out = self.full_field()
        self.lib.c2qo_m_tm_plus(out, inp, gauge, kappa, mubar)
        return out

    def m_tm_minus(self, inp, gauge, kappa, mubar):
        out = self.full_field()
        self.lib.c2qo_m_tm_minus(out, inp, gauge, kappa, mubar)
        return out

    def apply(self, op, inp, gauge, kappa, mubar, action=TWISTEDMASS, merged=False):
        out = self.eo_field()
        self.lib.c2qo_apply(op, out, inp, gauge, kappa, mubar, action, int(merged))
        return out

    # ---- solvers ----
    def cg(self, x, op, b, gauge, kappa, mubar, action=TWISTEDMASS, params=None):
        params = params or SolverParams(solver=1)
        return self.lib.c2qo_cg(x, op, b, gauge, kappa, mubar, action, C.byref(params))

    def bicgstab(self, x, op, b, gauge, kappa, mubar, action=TWISTEDMASS, params=None):
        params = params or SolverParams()
        return self.lib.c2qo_bicgstab(x, op, b, gauge, kappa, mubar, action, C.byref(params))

    def perform_inversion_eo(self, source, gauge, kappa, mubar, action=TWISTEDMASS, params=None):
        params = params or SolverParams()
        out = self.full_field()
        used = C.c_int(0)
        it = self.lib.c2qo_perform_inversion_eo(out, source, gauge, kappa, mubar, action, C.byref(params),
                                                C.byref(used))
        return out, it, bool(used.value)

    # ---- reference test fills ----
    # ---- HMC callers (gauge momenta: ae[4V], link mu + 4 site, 8 doubles) ----
    def gm_field(self):
        return np.zeros((4 * self.vol, 8))

    def fermion_force_eo(self, gm, Y, X, gauge, evenodd, kappa):
        """gm += the eo fermion force (in place)."""
        self.lib.c2qo_fermion_force_eo(gm, Y, X, gauge, evenodd, kappa)
        return gm

    def fermion_force_full(self, gm, Y, X, gauge, kappa):
        """gm += the non-eo fermion force of full fields Y, X (in place)."""
        self.lib.c2qo_fermion_force_full(gm, Y, X, gauge, kappa)
        return gm

    def gm_squarenorm(self, gm):
        return self.lib.c2qo_gm_squarenorm(gm)

    def calc_fermion_force_eo(self, gm, phi, gauge, kappa, mubar, action=TWISTEDMASS, params=None):
        params = params or SolverParams()
        return self.lib.c2qo_calc_fermion_force_eo(gm, phi, gauge, kappa, mubar, action, C.byref(params))

    def calc_s_fermion_eo(self, phi, gauge, kappa, mubar, action=TWISTEDMASS, params=None):
        params = params or SolverParams()
        it = C.c_int(0)
        s = self.lib.c2qo_calc_s_fermion_eo(phi, gauge, kappa, mubar, action, C.byref(params), C.byref(it))
        return s, it.value

    def pseudo_randomize(self, n_sites, seed):
        a = np.zeros((n_sites, 24))
        self.lib.c2qo_pseudo_randomize(a, a.size, seed)
        return a

    def gauge_fill(self, nontrivial):
        g = np.zeros((4 * self.vol, 18))
        self.lib.c2qo_fill_gauge(g, 4 * self.vol, int(nontrivial))
        return g

    def ascending_complex(self, n_sites):
        a = np.zeros((n_sites, 24))
        self.lib.c2qo_fill_ascending_complex(a, n_sites)
        return a

    def count_sf(self, a):
        return self.lib.c2qo_count_sf(np.ascontiguousarray(a), a.shape[0])

    # ---- the workload's seeded inputs (oracle_inputs.c) ----
    def gauge_generate(self, ns, nt, eps, seed):
        """U = exp(i eps H) per link, Matrixsu3[4V] (4*ns^3*nt, 18)."""
        g = np.empty((4 * ns ** 3 * nt, 18))
        if self.lib.c2qo_gauge_generate(g, ns, nt, eps, seed) != 0:
            raise ValueError("bad gauge generator arguments")
        return g

    def source_generate(self, n_sites, kind, seed):
        """kind "z2" or "gaussian": (n_sites, 24)."""
        out = np.empty((n_sites, 24))
        if self.lib.c2qo_source_generate(out, n_sites, {"z2": 0, "gaussian": 1}[kind], seed) != 0:
            raise ValueError("bad source generator arguments")
        return out


def available(kind: str) -> bool:
    name = {"port": "libc2q_oracle.so", "reference": "libc2q_ref.so"}[kind]
    return os.path.exists(os.path.join(_REF_DIR, name))
