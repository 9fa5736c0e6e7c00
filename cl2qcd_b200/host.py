"""Python mirror of the reference's host surface for the eo tm-Wilson inverter path.

Names, argument meaning and error behaviour follow CL2QCD:

* ``System``            -- hardware::System (hardware/system.cpp:117-200): one CUDA context/stream.
* ``Lattice``           -- nSpace/nTime/thetaFermion*/chemicalPotential* input parameters.
* ``Gaugefield``        -- physics::lattices::Gaugefield (physics/lattices/gaugefield.hpp:44-139).
* ``Spinorfield_eo``    -- physics::lattices::Spinorfield_eo (physics/lattices/spinorfield_eo.hpp:48-305),
  with the free BLAS functions saxpy (y - a x), sax, saxsbypz, scalar_product,
  squarenorm, saxpy_AND_squarenorm, saxpy_AND_gamma5_eo, copyData,
  convert_to_eoprec, convert_from_eoprec.
* ``dslash``, ``M_tm_*sitediagonal*`` -- physics::fermionmatrix explicit ops
  (physics/fermionmatrix/fermionmatrix.hpp:46-61).
* ``Aee``, ``Aee_minus``, ``Qplus_eo``, ``Qminus_eo``, ``QplusQminus_eo`` -- the eo
  fermion matrices (fermionmatrix.hpp:194-310), called as ``A(out, gf, in, params)``.
* ``cg``, ``bicgstab`` -- physics::algorithms::solvers (cg.hpp:41-56, bicgstab.hpp:42-57):
  return the iteration count, raise ``SolverStuck`` / ``SolverDidNotSolve``
  (physics/algorithms/solvers/exceptions.hpp:35-62).
* ``perform_inversion`` -- physics::algorithms::perform_inversion, eo branch (inversion.cpp:44-242).
* ``Gaugemomenta``, ``fermion_force``, ``calc_fermion_force``, ``calc_s_fermion`` -- the
  HMC callers of the eo solvers (physics/lattices/gaugemomenta.hpp,
  physics/algorithms/fermion_force.cpp, physics/algorithms/metropolis.cpp).

Everything runs in the CUDA library; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib as L


class SolverException(RuntimeError):
    """physics::algorithms::solvers::SolverException"""

    def __init__(self, iterations, msg=""):
        super().__init__(msg or self.__class__.__name__)
        self.iterations = iterations


class SolverStuck(SolverException):
    pass


class SolverDidNotSolve(SolverException):
    pass


class InvalidParameters(ValueError):
    """Invalid_Parameters / std::invalid_argument of the reference."""


def _check(rc, ctx=None, lib=None):
    if rc >= 0:
        return rc
    msg = ""
    if ctx is not None and lib is not None:
        msg = (lib.c2q_last_error(ctx) or b"").decode()
    if rc == L.BAD_ARG:
        raise InvalidParameters(msg)
    raise L.C2QError(rc, msg)


class System:
    """One device context (hardware::System with one device)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.lib = L.load()
        h = C.c_void_p()
        rc = self.lib.c2q_ctx_create(C.byref(h), device, C.c_void_p(stream) if stream else None)
        if rc != 0:
            raise L.C2QError(rc, "c2q_ctx_create failed (no CUDA device?)")
        self.h = h
        # device objects of this context; they are destroyed before the context
        self._children = weakref.WeakSet()

    def _adopt(self, obj):
        self._children.add(obj)

    def synchronize(self):
        _check(self.lib.c2q_ctx_synchronize(self.h), self.h, self.lib)

    @property
    def launch_count(self) -> int:
        return self.lib.c2q_ctx_launch_count(self.h)

    def set_link_format(self, rec12: bool):
        """Links read by the explicit operator calls: 18-real (default) or 12-real."""
        _check(self.lib.c2q_ctx_set_link_format(self.h, int(bool(rec12))), self.h, self.lib)

    def set_sweep_choice(self, choice: int):
        """Pin the launch choice of the reduced-precision sweeps (-1: the autotuner's)."""
        _check(self.lib.c2q_ctx_set_sweep_choice(self.h, choice), self.h, self.lib)

    def tune_report(self) -> str:
        """The launch configurations the autotuner chose, one line per launch shape."""
        n = self.lib.c2q_ctx_tune_report(self.h, None, 0)
        buf = C.create_string_buffer(max(n, 1))
        self.lib.c2q_ctx_tune_report(self.h, buf, len(buf))
        return buf.value.decode()

    def close(self):
        if getattr(self, "h", None):
            for child in list(self._children):
                child._destroy()
            self.lib.c2q_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass(frozen=True)
class Lattice:
    """nSpace, nTime, thetaFermionTemporal/Spatial (units of pi), chemical potential."""

    ns: int
    nt: int
    theta_t: float = 0.0
    theta_s: float = 0.0
    cp_re: float | None = None
    cp_im: float | None = None

    def c(self) -> L.CLattice:
        return L.CLattice(self.ns, self.nt, self.theta_t, self.theta_s, int(self.cp_re is not None),
                          int(self.cp_im is not None), self.cp_re or 0.0, self.cp_im or 0.0)

    @property
    def vol(self):
        return self.ns ** 3 * self.nt

    @property
    def seo(self):
        return self.vol // 2


@dataclass
class AdditionalParameters:
    """physics::AdditionalParameters: kappa and mubar = 2 kappa mu (meta/util.cpp:56-59)."""

    kappa: float
    mubar: float = 0.0

    @classmethod
    def from_mu(cls, kappa, mu):
        return cls(kappa, 2.0 * kappa * mu)


class Gaugefield:
    def __init__(self, system: System, lattice: Lattice, aos: np.ndarray | None = None):
        self.system, self.lattice = system, lattice
        lib = system.lib
        h = C.c_void_p()
        lc = lattice.c()
        _check(lib.c2q_gauge_create(system.h, C.byref(lc), C.byref(h)), system.h, lib)
        self.h = h
        system._adopt(self)
        if aos is not None:
            self.upload(aos)

    def upload(self, aos):
        aos = np.ascontiguousarray(aos, dtype=np.float64)
        assert aos.size == 4 * self.lattice.vol * 18
        _check(self.system.lib.c2q_gauge_upload(self.h, aos.reshape(-1)), self.system.h, self.system.lib)

    def download(self):
        out = np.zeros(4 * self.lattice.vol * 18)
        _check(self.system.lib.c2q_gauge_download(self.h, out), self.system.h, self.system.lib)
        return out.reshape(4 * self.lattice.vol, 18)

    @property
    def device_bytes(self):
        return self.system.lib.c2q_gauge_device_bytes(self.h)

    def unitarity(self) -> dict:
        """FP64 distance of the uploaded links from SU(3), measured on the device:
        max |U U^dagger - 1| (entry-wise), max |det U - 1|, and max |row 2 -
        conj(row0 x row1)| (what 12-real storage changes)."""
        dev = (C.c_double * 3)()
        _check(self.system.lib.c2q_gauge_unitarity(self.h, dev), self.system.h, self.system.lib)
        return {"unitarity": dev[0], "det": dev[1], "rec12": dev[2]}

    def reunitarize(self) -> float:
        """project_su3 (ocl_kernel/operations_gaugefield.cl:135-240) on every link
        in FP64 on the device; returns max |U U^dagger - 1| before the projection."""
        before = C.c_double()
        _check(self.system.lib.c2q_gauge_reunitarize(self.h, C.byref(before)), self.system.h, self.system.lib)
        return before.value

    def _destroy(self):
        # a context outlives its objects: nothing to do once the context is closed
        if getattr(self, "h", None) and getattr(self.system, "h", None):
            self.system.lib.c2q_gauge_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass


class Spinorfield_eo:
    """An eo spinor field.  `precision` 64 is the reference's; 32 / 16 are the
    reduced-precision storages of the mixed solvers (NT a multiple of 4)."""

    def __init__(self, system: System, lattice: Lattice, aos: np.ndarray | None = None, precision: int = 64):
        self.system, self.lattice = system, lattice
        self.precision = precision
        lib = system.lib
        h = C.c_void_p()
        lc = lattice.c()
        _check(lib.c2q_spinor_eo_create_precision(system.h, C.byref(lc), precision, C.byref(h)), system.h, lib)
        self.h = h
        system._adopt(self)
        if aos is not None:
            self.load(aos)

    # Spinor::load / dump
    def load(self, aos):
        aos = np.ascontiguousarray(aos, dtype=np.float64).reshape(-1)
        assert aos.size == self.lattice.seo * 24
        _check(self.system.lib.c2q_spinor_eo_upload(self.h, aos), self.system.h, self.system.lib)

    def dump(self):
        out = np.zeros(self.lattice.seo * 24)
        _check(self.system.lib.c2q_spinor_eo_download(self.h, out), self.system.h, self.system.lib)
        return out.reshape(self.lattice.seo, 24)

    def zero(self):
        _check(self.system.lib.c2q_spinor_eo_zero(self.h), self.system.h, self.system.lib)

    def cold(self):
        _check(self.system.lib.c2q_spinor_eo_cold(self.h), self.system.h, self.system.lib)

    def gamma5(self):
        _check(self.system.lib.c2q_gamma5_eo(self.h), self.system.h, self.system.lib)

    def convert_from(self, other: "Spinorfield_eo"):
        """self = other rounded (or widened) to this field's precision."""
        _check(self.system.lib.c2q_spinor_eo_convert(self.h, other.h), self.system.h, self.system.lib)

    def _destroy(self):
        if getattr(self, "h", None) and getattr(self.system, "h", None):
            self.system.lib.c2q_spinor_eo_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass


def _sys(f):
    return f.system


def _c(rc, f):
    return _check(rc, f.system.h, f.system.lib)


# ---------------- eo BLAS (physics/lattices/spinorfield_eo.hpp) ----------------
def saxpy(out, alpha, x, y):
    """out = y - alpha x"""
    a = complex(alpha)
    _c(out.system.lib.c2q_saxpy(out.h, a.real, a.imag, x.h, y.h), out)


def saxpy_AND_gamma5_eo(out, alpha, x, y):
    a = complex(alpha)
    _c(out.system.lib.c2q_saxpy_AND_gamma5_eo(out.h, a.real, a.imag, x.h, y.h), out)


def sax(out, alpha, x):
    a = complex(alpha)
    _c(out.system.lib.c2q_sax(out.h, a.real, a.imag, x.h), out)


def saxsbypz(out, alpha, x, beta, y, z):
    a, b = complex(alpha), complex(beta)
    _c(out.system.lib.c2q_saxsbypz(out.h, a.real, a.imag, x.h, b.real, b.imag, y.h, z.h), out)


def copyData(to, frm):
    _c(to.system.lib.c2q_copyData(to.h, frm.h), to)


def scalar_product(x, y) -> complex:
    re, im = C.c_double(), C.c_double()
    _c(x.system.lib.c2q_scalar_product(x.h, y.h, C.byref(re), C.byref(im)), x)
    return complex(re.value, im.value)


def squarenorm(x) -> float:
    """squarenorm of an eo spinor field, or of gauge momenta (the reference's overload)."""
    r = C.c_double()
    if isinstance(x, Gaugemomenta):
        _c(x.system.lib.c2q_gaugemomenta_squarenorm(x.h, C.byref(r)), x)
    else:
        _c(x.system.lib.c2q_squarenorm(x.h, C.byref(r)), x)
    return r.value


def saxpy_AND_squarenorm(out, alpha, x, y) -> float:
    a = complex(alpha)
    r = C.c_double()
    _c(out.system.lib.c2q_saxpy_AND_squarenorm(out.h, a.real, a.imag, x.h, y.h, C.byref(r)), out)
    return r.value


def convert_to_eoprec(even, odd, full):
    full = np.ascontiguousarray(full, dtype=np.float64).reshape(-1)
    _c(even.system.lib.c2q_convert_to_eoprec(even.h, odd.h, full), even)


def convert_from_eoprec(even, odd) -> np.ndarray:
    out = np.zeros(even.lattice.vol * 24)
    _c(even.system.lib.c2q_convert_from_eoprec(out, even.h, odd.h), even)
    return out.reshape(even.lattice.vol, 24)


# ---------------- explicit fermion ops (physics/fermionmatrix/explicit.cpp) ----------------
EVEN, ODD = L.EVEN, L.ODD


def dslash(out, gf, in_, evenodd, kappa):
    _c(out.system.lib.c2q_dslash_eo(out.h, gf.h, in_.h, evenodd, kappa), out)


def dslash_AND_M_tm_inverse_sitediagonal(out, gf, in_, evenodd, kappa, mubar, minus=False):
    _c(out.system.lib.c2q_dslash_AND_M_tm_inverse_sitediagonal_eo(out.h, gf.h, in_.h, evenodd, kappa, mubar,
                                                                  int(minus)), out)


def _diag(which):
    def f(out, in_, mubar):
        _c(out.system.lib.c2q_tm_sitediagonal(out.h, in_.h, mubar, which), out)

    return f


M_tm_sitediagonal = _diag(L.DIAG_M_TM)
M_tm_inverse_sitediagonal = _diag(L.DIAG_M_TM_INVERSE)
M_tm_sitediagonal_minus = _diag(L.DIAG_M_TM_MINUS)
M_tm_inverse_sitediagonal_minus = _diag(L.DIAG_M_TM_INVERSE_MINUS)
M_tm_sitediagonal_AND_gamma5_eo = _diag(L.DIAG_M_TM_AND_GAMMA5)
M_tm_sitediagonal_minus_AND_gamma5_eo = _diag(L.DIAG_M_TM_MINUS_AND_GAMMA5)


# ---------------- eo fermion matrices ----------------
class Fermionmatrix_eo:
    OP = None

    def __init__(self, action: str = "twistedmass", merged: bool = False):
        act = action.lower()
        if act not in ("wilson", "twistedmass"):
            raise InvalidParameters("Unkown fermion action! (wilson or twistedmass)")
        self.action = L.WILSON if act == "wilson" else L.TWISTEDMASS
        self.merged = merged

    def __call__(self, out, gf, in_, params: AdditionalParameters):
        _c(out.system.lib.c2q_apply_eo(self.OP, out.h, gf.h, in_.h, params.kappa, params.mubar, self.action,
                                       int(self.merged)), out)


class Aee(Fermionmatrix_eo):
    OP = L.OP_AEE


class Aee_minus(Fermionmatrix_eo):
    OP = L.OP_AEE_MINUS


class Aee_AND_gamma5_eo(Fermionmatrix_eo):
    OP = L.OP_AEE_AND_GAMMA5_EO


class Aee_minus_AND_gamma5_eo(Fermionmatrix_eo):
    OP = L.OP_AEE_MINUS_AND_GAMMA5_EO


class Qplus_eo(Fermionmatrix_eo):
    OP = L.OP_QPLUS_EO


class Qminus_eo(Fermionmatrix_eo):
    OP = L.OP_QMINUS_EO


class QplusQminus_eo(Fermionmatrix_eo):
    OP = L.OP_QPLUSQMINUS_EO


# ---------------- solvers ----------------
@dataclass
class SolverParameters:
    """SolversParametersInterface (defaults of meta/parametersSolver.cpp:74-107) plus the
    precision/reliable-update/rel_tol extensions of this build."""

    solver: str = "bicgstab"
    prec: float = 1e-23
    rel_tol: float = 0.0
    cgmax: int = 1000
    iter_refresh: int = 100
    resid_check_every: int = 10
    min_iter: int = 0
    precision: int = 64
    reliable_delta: float = 0.003
    use_rec12: bool = False
    use_graph: bool = False
    temporal_gauge: bool = True

    def c(self) -> L.CSolverParams:
        s = {"cg": L.SOLVER_CG, "bicgstab": L.SOLVER_BICGSTAB, "bicgstab_save": L.SOLVER_BICGSTAB_SAVE}
        if self.solver not in s:
            raise InvalidParameters(f"unknown solver {self.solver}")
        return L.CSolverParams(s[self.solver], self.prec, self.rel_tol, self.cgmax, self.iter_refresh,
                               self.resid_check_every, self.min_iter, self.precision, self.reliable_delta,
                               int(self.use_rec12), int(self.use_graph), int(self.temporal_gauge))


def _solve(fn, x, A, gf, b, params, add, report, fn_full=None):
    lib = x.system.lib
    p = params.c()
    rep = L.CSolveReport()
    if isinstance(x, Spinorfield):  # full fields (useEO=false): a full-lattice matrix
        rc = fn_full(x.even.h, x.odd.h, A.OP, gf.h, b.even.h, b.odd.h, add.kappa, add.mubar, A.action,
                     C.byref(p), C.byref(rep))
    else:
        rc = fn(x.h, A.OP, gf.h, b.h, add.kappa, add.mubar, A.action, C.byref(p), C.byref(rep))
    if report is not None:
        report.update(rep.as_dict())
    if rc == L.SOLVER_STUCK:
        raise SolverStuck(rep.iterations, (lib.c2q_last_error(x.system.h) or b"").decode())
    if rc == L.DID_NOT_SOLVE:
        raise SolverDidNotSolve(rep.iterations, (lib.c2q_last_error(x.system.h) or b"").decode())
    return _check(rc, x.system.h, lib)


def cg(x, A, gf, b, params: SolverParameters, add: AdditionalParameters, report: dict | None = None) -> int:
    """solvers::cg on eo fields (A an eo matrix) or on full fields (A a full-lattice matrix)."""
    return _solve(x.system.lib.c2q_cg, x, A, gf, b, params, add, report, x.system.lib.c2q_cg_full)


def cg_multi(xs, A, gf, bs, params: SolverParameters, add: AdditionalParameters,
             reports: list | None = None) -> list:
    """CG on A x[k] = b[k] for every k.  With precision 32 or 16 up to 16
    right-hand sides iterate as one batch whose sweeps read each link once;
    each right-hand side keeps its own scalars, reliable updates and stopping
    test (the same semantics as cg).  Returns the iteration counts."""
    n = len(xs)
    assert n == len(bs) and n > 0
    lib = xs[0].system.lib
    p = params.c()
    ax = (C.c_void_p * n)(*[x.h for x in xs])
    ab = (C.c_void_p * n)(*[b.h for b in bs])
    reps = (L.CSolveReport * n)()
    rc = lib.c2q_cg_multi(ax, A.OP, gf.h, ab, n, add.kappa, add.mubar, A.action, C.byref(p), reps)
    out = [r.as_dict() for r in reps]
    if reports is not None:
        reports.clear()
        reports.extend(out)
    msg = (lib.c2q_last_error(xs[0].system.h) or b"").decode()
    if rc == L.SOLVER_STUCK:
        raise SolverStuck(max(r["iterations"] for r in out), msg)
    if rc == L.DID_NOT_SOLVE:
        raise SolverDidNotSolve(max(r["iterations"] for r in out), msg)
    _check(rc, xs[0].system.h, lib)
    return [r["iterations"] for r in out]


def point_source(n_sites: int, k: int) -> np.ndarray:
    """Spin-colour point source k (spin k % 4, colour k // 4) at the origin, as
    an eo field: the origin is eo site 0 of the even sites
    (ocl_kernel/operations_geometry.cl:476-489, spinorfield_point_source.cl:23-75)."""
    out = np.zeros((n_sites, 24))
    spin, colour = k % 4, k // 4
    out[0, 2 * (3 * spin + colour)] = 1.0
    return out


def bicgstab(x, A, gf, b, params: SolverParameters, add: AdditionalParameters, report: dict | None = None) -> int:
    """solvers::bicgstab on eo fields (A an eo matrix) or on full fields (A a full-lattice matrix).
    On eo fields, params.precision 32 or 16 runs it on FP32 / FP16 fields with FP64 reliable
    updates (report["reliable_updates"] counts them); full fields are FP64."""
    return _solve(x.system.lib.c2q_bicgstab, x, A, gf, b, params, add, report, x.system.lib.c2q_bicgstab_full)


def perform_inversion(system: System, gf: Gaugefield, source: np.ndarray, params: SolverParameters,
                      add: AdditionalParameters, action: str = "twistedmass", report: dict | None = None,
                      use_eo: bool = True):
    """One source of perform_inversion; returns the full result field.  use_eo
    (the reference's useEO): the eo Schur solve with the reference's sign
    convention (inversion.cpp:123-236), else the full-lattice solve
    (inversion.cpp:98-122, result = M^-1 source)."""
    lib = system.lib
    src = np.ascontiguousarray(source, dtype=np.float64).reshape(-1)
    out = np.zeros_like(src)
    p = params.c()
    rep = L.CSolveReport()
    act = L.WILSON if action.lower() == "wilson" else L.TWISTEDMASS
    fn = lib.c2q_perform_inversion_eo if use_eo else lib.c2q_perform_inversion_full
    rc = fn(system.h, out, gf.h, src, add.kappa, add.mubar, act, C.byref(p), C.byref(rep))
    if report is not None:
        report.update(rep.as_dict())
    if rc == L.SOLVER_STUCK:
        raise SolverStuck(rep.iterations)
    if rc == L.DID_NOT_SOLVE:
        raise SolverDidNotSolve(rep.iterations)
    _check(rc, system.h, lib)
    return out.reshape(gf.lattice.vol, 24), rc


def point_source_full(lattice: Lattice, k: int, x: int = 0, y: int = 0, z: int = 0, t: int = 0) -> np.ndarray:
    """Full-field point source k (spin k % 4, colour k // 4, content "one") at
    (x, y, z, t) (spinorfield_point_source.cl:23-75, physics/sources.cpp:35-60)."""
    out = np.zeros((lattice.vol, 24))
    site = x + lattice.ns * (y + lattice.ns * (z + lattice.ns * t))
    out[site, 2 * (3 * (k % 4) + k // 4)] = 1.0
    return out


def inverter_ps_correlator(system: System, gf: Gaugefield, params: SolverParameters, add: AdditionalParameters,
                           n_sources: int = 12, position=(0, 0, 0, 0), action: str = "twistedmass",
                           reports: list | None = None, direction: int = 3, use_eo: bool = True) -> np.ndarray:
    """The inverter's point-source measurement (physics/observables/wilsonTwoFlavourCorrelators.cpp:
    measureTwoFlavourDoubletCorrelatorsOnGaugefieldAndWriteToFile with the default 12 point
    sources): perform_inversion of each spin-colour point source (eo, results kept on the
    device; or, use_eo False, the full-lattice solve), and the pseudoscalar correlator
    contracted on the GPU along z (direction 3, the reference's default correlatorDirection)
    or t (direction 0)."""
    lib = system.lib
    L_ = gf.lattice
    act = L.WILSON if action.lower() == "wilson" else L.TWISTEDMASS
    evens = [Spinorfield_eo(system, L_) for _ in range(n_sources)]
    odds = [Spinorfield_eo(system, L_) for _ in range(n_sources)]
    p = params.c()
    for k in range(n_sources):
        src = point_source_full(L_, k % 12, *position).reshape(-1)
        rep = L.CSolveReport()
        if use_eo:
            rc = lib.c2q_perform_inversion_eo_fields(system.h, evens[k].h, odds[k].h, gf.h, src, add.kappa,
                                                     add.mubar, act, C.byref(p), C.byref(rep))
        else:
            res = np.zeros_like(src)
            rc = lib.c2q_perform_inversion_full(system.h, res, gf.h, src, add.kappa, add.mubar, act, C.byref(p),
                                                C.byref(rep))
            if rc >= 0:
                _check(lib.c2q_convert_to_eoprec(evens[k].h, odds[k].h, res), system.h, lib)
        if reports is not None:
            reports.append(rep.as_dict())
        if rc == L.SOLVER_STUCK:
            raise SolverStuck(rep.iterations)
        if rc == L.DID_NOT_SOLVE:
            raise SolverDidNotSolve(rep.iterations)
        _check(rc, system.h, lib)
    out = np.zeros(L_.nt if direction == 0 else L_.ns)
    ae = (C.c_void_p * n_sources)(*[f.h for f in evens])
    ao = (C.c_void_p * n_sources)(*[f.h for f in odds])
    _check(lib.c2q_correlator_ps(ae, ao, n_sources, add.kappa, direction, out), system.h, lib)
    return out


def read_ildg(path: str):
    """A gauge configuration in ILDG/LIME format (the reference's ildg_io reader):
    returns (ns, nt, Matrixsu3[4V] as float64 (4V, 18), info) with info holding the
    precision, the xlf-info text and the SciDAC checksum (computed, and whether it
    matches the recorded one: 1 yes, 0 no, -1 not recorded)."""
    lib = L.load()
    ns, nt, prec, st = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    a, b = C.c_uint(), C.c_uint()
    p = path.encode()
    _check(lib.c2q_ildg_read(p, None, 0, C.byref(ns), C.byref(nt), C.byref(prec), None, 0, None, None, None))
    aos = np.zeros((4 * ns.value ** 3 * nt.value, 18))
    text = C.create_string_buffer(4096)
    _check(lib.c2q_ildg_read(p, aos.ctypes.data, aos.size, C.byref(ns), C.byref(nt), C.byref(prec), text, 4096,
                             C.byref(a), C.byref(b), C.byref(st)))
    info = {"precision": prec.value, "xlf_info": text.value.decode(errors="replace"), "suma": a.value,
            "sumb": b.value, "checksum_status": st.value}
    return ns.value, nt.value, aos, info


def plaquette(lattice: Lattice, aos: np.ndarray) -> float:
    """Average plaquette (1/3) Re tr U_mu(x) U_nu(x+mu) U_mu(x+nu)^+ U_nu(x)^+ over the
    6 planes and all sites, from a host Matrixsu3[4V] (mu 0 = time)."""
    ns, nt = lattice.ns, lattice.nt
    U = aos.reshape(nt, ns, ns, ns, 4, 3, 3, 2)  # [t][z][y][x][mu][row][col][re,im]
    U = U[..., 0] + 1j * U[..., 1]
    axis = {0: 0, 1: 3, 2: 2, 3: 1}  # direction -> array axis (t, z, y, x)
    tot = 0.0
    for mu in range(4):
        for nu in range(mu + 1, 4):
            a = U[..., mu, :, :]
            b = np.roll(U[..., nu, :, :], -1, axis=axis[mu])
            c = np.roll(U[..., mu, :, :], -1, axis=axis[nu])
            d = U[..., nu, :, :]
            p_ = a @ b @ np.conj(np.swapaxes(c, -1, -2)) @ np.conj(np.swapaxes(d, -1, -2))
            tot += np.trace(p_, axis1=-2, axis2=-1).real.sum()
    return tot / (6 * 3 * lattice.vol)


# ---------------- inputs ----------------
def generate_gaugefield(lattice: Lattice, eps: float, seed: int) -> np.ndarray:
    """U = exp(i eps H), reunitarised (host, library code)."""
    lib = L.load()
    out = np.zeros(4 * lattice.vol * 18)
    _check(lib.c2q_gauge_generate(out, lattice.ns, lattice.nt, eps, seed))
    return out.reshape(4 * lattice.vol, 18)


def generate_source(n_sites: int, kind: str, seed: int) -> np.ndarray:
    lib = L.load()
    out = np.zeros(n_sites * 24)
    _check(lib.c2q_source_generate(out, n_sites, {"z2": 0, "gaussian": 1}[kind], seed))
    return out.reshape(n_sites, 24)


# ---------------- full-lattice fields and operators ----------------
class Spinorfield:
    """physics::lattices::Spinorfield (a full-lattice field, physics/lattices/spinorfield.hpp),
    held on the device as its two parities (even = sites with x+y+z+t even)."""

    def __init__(self, system: System, lattice: Lattice, aos: np.ndarray | None = None, precision: int = 64):
        self.system, self.lattice = system, lattice
        self.even = Spinorfield_eo(system, lattice, precision=precision)
        self.odd = Spinorfield_eo(system, lattice, precision=precision)
        if aos is not None:
            self.load(aos)

    def load(self, aos):
        aos = np.ascontiguousarray(aos, dtype=np.float64).reshape(-1)
        assert aos.size == self.lattice.vol * 24
        _check(self.system.lib.c2q_convert_to_eoprec(self.even.h, self.odd.h, aos), self.system.h, self.system.lib)

    def dump(self):
        out = np.zeros(self.lattice.vol * 24)
        _check(self.system.lib.c2q_convert_from_eoprec(out, self.even.h, self.odd.h), self.system.h, self.system.lib)
        return out.reshape(self.lattice.vol, 24)


class Fermionmatrix:
    """Full-lattice fermion matrices (physics/fermionmatrix/fermionmatrix.hpp, non-eo)."""
    OP = None

    def __init__(self, action: str = "twistedmass"):
        self.action = L.WILSON if action.lower() == "wilson" else L.TWISTEDMASS

    def __call__(self, out: Spinorfield, gf, in_: Spinorfield, params: AdditionalParameters):
        sysm = out.system
        _check(sysm.lib.c2q_apply_full(self.OP, out.even.h, out.odd.h, gf.h, in_.even.h, in_.odd.h, params.kappa,
                                       params.mubar, self.action), sysm.h, sysm.lib)


class M_tm_plus(Fermionmatrix):
    OP = L.FULL_M_TM_PLUS


class M_tm_minus(Fermionmatrix):
    OP = L.FULL_M_TM_MINUS


class Qplus(Fermionmatrix):
    OP = L.FULL_QPLUS


class Qminus(Fermionmatrix):
    OP = L.FULL_QMINUS


class QplusQminus(Fermionmatrix):
    OP = L.FULL_QPLUSQMINUS


def M_wilson(out: Spinorfield, gf, in_: Spinorfield, kappa: float):
    """physics::fermionmatrix::M_wilson (explicit.cpp): (1 - kappa D) in."""
    Fermionmatrix.__call__(M_tm_plus("wilson"), out, gf, in_, AdditionalParameters(kappa, 0.0))


def squarenorm_full(x: Spinorfield) -> float:
    return squarenorm(x.even) + squarenorm(x.odd)


# ---------------- serving (no counterpart in the reference) ----------------
class Server:
    """Request loop on one GPU (c2q_server_*): `slots` worker threads with their
    own streams; requests are admitted as soon as a slot and HBM (by
    footprint) are free, so their work overlaps on the device; gauge fields are
    registered once and stay resident.  Each request solves QplusQminus_eo for
    `nsrc` seeded sources (generated on the device) with the multi-right-hand-
    side mixed-precision CG."""

    def __init__(self, device: int = 0, slots: int = 2, hbm_budget: int = 0, precision: int = 16,
                 rec12: bool = True):
        self.lib = L.load()
        h = C.c_void_p()
        _check(self.lib.c2q_server_create(C.byref(h), device, slots, hbm_budget, precision, int(rec12)))
        self.h = h
        self._keep = {}

    def set_heavy_limit(self, heavy_site_rhs: int, max_heavy: int):
        """At most `max_heavy` requests with eo sites x sources >= heavy_site_rhs run
        at a time (default 2^19 and 1); lighter requests are admitted beside them."""
        _check(self.lib.c2q_server_set_heavy_limit(self.h, heavy_site_rhs, max_heavy))

    def add_gauge(self, gauge_id: int, lattice: Lattice, aos: np.ndarray):
        aos = np.ascontiguousarray(aos, dtype=np.float64).reshape(-1)
        lc = lattice.c()
        _check(self.lib.c2q_server_add_gauge(self.h, gauge_id, C.byref(lc), aos))

    def submit(self, lattice: Lattice, gauge_id: int, kappa: float, mu: float, nsrc: int, seed: int,
               source_kind: str = "z2", params: SolverParameters | None = None,
               solutions: np.ndarray | None = None) -> int:
        """Queue a request; `solutions` (optional, float64 (nsrc, Seo, 24)) receives the solutions."""
        params = params or SolverParameters(solver="cg", prec=0.0, rel_tol=1e-10, cgmax=40000)
        r = L.CRequest()
        r.lat = lattice.c()
        r.gauge_id = gauge_id
        r.kappa, r.mu = kappa, mu
        r.nsrc = nsrc
        r.source_kind = {"z2": 0, "gaussian": 1}[source_kind]
        r.source_seed = seed
        r.params = params.c()
        r.solutions = solutions.ctypes.data if solutions is not None else None
        t = C.c_longlong()
        _check(self.lib.c2q_server_submit(self.h, C.byref(r), C.byref(t)))
        if solutions is not None:
            self._keep[t.value] = solutions
        return t.value

    def wait(self, ticket: int) -> dict:
        res = L.CRequestResult()
        _check(self.lib.c2q_server_wait(self.h, ticket, C.byref(res)))
        self._keep.pop(ticket, None)
        return res.as_dict()

    def stats(self) -> dict:
        st = L.CServerStats()
        _check(self.lib.c2q_server_get_stats(self.h, C.byref(st)))
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.lib.c2q_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def request_footprint(lattice: Lattice, nsrc: int, precision: int = 16) -> int:
    """Device bytes a serving request holds while it runs (its admission footprint)."""
    lc = lattice.c()
    return L.load().c2q_request_footprint(C.byref(lc), nsrc, precision)


# ---------------- HMC callers of the eo solvers ----------------
class Gaugemomenta:
    """physics::lattices::Gaugemomenta: 8 reals (the su(3) algebra element) per
    link; host format ae[4V] at link mu + 4 site."""

    def __init__(self, system: System, lattice: Lattice, aos: np.ndarray | None = None):
        self.system, self.lattice = system, lattice
        lib = system.lib
        h = C.c_void_p()
        lc = lattice.c()
        _check(lib.c2q_gaugemomenta_create(system.h, C.byref(lc), C.byref(h)), system.h, lib)
        self.h = h
        system._adopt(self)
        if aos is not None:
            self.upload(aos)

    def zero(self):
        _c(self.system.lib.c2q_gaugemomenta_zero(self.h), self)

    def upload(self, aos):
        aos = np.ascontiguousarray(aos, dtype=np.float64)
        assert aos.size == 4 * self.lattice.vol * 8
        _c(self.system.lib.c2q_gaugemomenta_upload(self.h, aos.reshape(-1)), self)

    def download(self):
        out = np.zeros(4 * self.lattice.vol * 8)
        _c(self.system.lib.c2q_gaugemomenta_download(self.h, out), self)
        return out.reshape(4 * self.lattice.vol, 8)

    def _destroy(self):
        if getattr(self, "h", None) and getattr(self.system, "h", None):
            self.system.lib.c2q_gaugemomenta_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass


def fermion_force(gm: Gaugemomenta, Y, X, *args):
    """physics::algorithms::fermion_force, both overloads:
    fermion_force(gm, Y, X, evenodd, gf, add) on eo fields (fermion_force.cpp:699-730):
    gm += the force of Y (on the sites evenodd selects: ODD the even ones) and X;
    fermion_force(gm, Y, X, gf, add) on full fields (fermion_force.cpp:672-697,
    force_fermion.cl): the same sum over every site, i.e. the eo force of both parities."""
    lib = gm.system.lib
    if isinstance(Y, Spinorfield):
        gf, add = args
        _c(lib.c2q_fermion_force_eo(gm.h, gf.h, Y.even.h, X.odd.h, ODD, add.kappa), gm)
        _c(lib.c2q_fermion_force_eo(gm.h, gf.h, Y.odd.h, X.even.h, EVEN, add.kappa), gm)
    else:
        evenodd, gf, add = args
        _c(lib.c2q_fermion_force_eo(gm.h, gf.h, Y.h, X.h, evenodd, add.kappa), gm)


def _odd_partner(out, tmp, gf, field, add, action, minus):
    """out = -M^-1 D(ODD) field (tm; -D(ODD) field for Wilson), fermion_force.cpp:144-175."""
    dslash(out, gf, field, ODD, add.kappa)
    if action == "twistedmass":
        (M_tm_inverse_sitediagonal_minus if minus else M_tm_inverse_sitediagonal)(tmp, out, add.mubar)
        sax(out, -1.0, tmp)
    else:
        sax(out, -1.0, out)


def calc_fermion_force(force: Gaugemomenta, gf: Gaugefield, phi, params: SolverParameters,
                       add: AdditionalParameters, action: str = "twistedmass", report: dict | None = None) -> int:
    """physics::algorithms::calc_fermion_force on eo fields, CG branch
    (fermion_force.cpp:37-80, 131-175): X = (Q+Q-)^-1 phi from a cold start,
    Y = Q- X, force += F(Y, X_odd, EVEN) + F(Y_odd, X, ODD).  The solve takes
    `params` (FP64 with the reference's semantics, or the mixed-precision CG).
    Returns the CG's iteration count."""
    system, lat = phi.system, phi.lattice
    x = Spinorfield_eo(system, lat)
    y = Spinorfield_eo(system, lat)
    tmp1 = Spinorfield_eo(system, lat)
    tmp2 = Spinorfield_eo(system, lat)
    x.cold()
    it = cg(x, QplusQminus_eo(action), gf, phi, params, add, report)
    Qminus_eo(action)(y, gf, x, add)
    _odd_partner(tmp1, tmp2, gf, x, add, action, minus=True)
    fermion_force(force, y, tmp1, EVEN, gf, add)
    _odd_partner(tmp1, tmp2, gf, y, add, action, minus=False)
    fermion_force(force, tmp1, x, ODD, gf, add)
    return it


def calc_s_fermion(gf: Gaugefield, phi, params: SolverParameters, add: AdditionalParameters,
                   action: str = "twistedmass", report: dict | None = None) -> float:
    """physics::algorithms::calc_s_fermion on eo fields, CG branch (metropolis.cpp:79-121):
    X = (Q+Q-)^-1 phi from a cold start, S_f = |Q- X|^2."""
    system, lat = phi.system, phi.lattice
    x = Spinorfield_eo(system, lat)
    y = Spinorfield_eo(system, lat)
    x.cold()
    cg(x, QplusQminus_eo(action), gf, phi, params, add, report)
    Qminus_eo(action)(y, gf, x, add)
    return squarenorm(y)
