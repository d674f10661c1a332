"""ctypes wrapper around the CPU checkers (test infrastructure only).

Two libraries expose the same calls:

* ``_ref/libsdddst_ref.so``  -- the reference hot path compiled in place
  (``oracle/Makefile``, target ``ref``) with ``ref_harness.cpp``;
* ``_build/libsdddst_oracle.so`` -- the project's C restatement
  ``sdddst_oracle.c`` (target ``port``).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libsdddst_ref.so")
PORT_LIB = os.path.join(HERE, "_build", "libsdddst_oracle.so")


class RefParams(C.Structure):
    _fields_ = [
        ("cutoff_multiplier", C.c_double),
        ("prec", C.c_double),
        ("step_size", C.c_double),
        ("stress_kind", C.c_int),
        ("stress_rate", C.c_double),
        ("spring_constant", C.c_double),
        ("stress_value", C.c_double),
        ("pd_scaling", C.c_int),
        ("calculate_strain", C.c_int),
        ("order_parameter", C.c_int),
        ("max_step_limited", C.c_int),
        ("max_step", C.c_double),
    ]


_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

_libs = {}


def _load(path: str):
    if path in _libs:
        return _libs[path]
    lib = C.CDLL(path)
    lib.ref_create.restype = C.c_void_p
    lib.ref_create.argtypes = [C.c_int, _D, C.c_int, C.c_void_p, C.POINTER(RefParams)]
    lib.ref_destroy.argtypes = [C.c_void_p]
    lib.ref_get_params.argtypes = [C.c_void_p, _D]
    lib.ref_step.argtypes = [C.c_void_p]
    lib.ref_step.restype = C.c_int
    lib.ref_get_scalars.argtypes = [C.c_void_p, _D]
    lib.ref_get_config.argtypes = [C.c_void_p, C.c_int, _D]
    lib.ref_get_vector.argtypes = [C.c_void_p, C.c_int, _D]
    lib.ref_set_state.argtypes = [C.c_void_p, _D, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
    lib.ref_speeds.argtypes = [C.c_void_p, _D, C.c_double, C.c_int, _D, _D]
    lib.ref_jacobian.restype = C.c_long
    lib.ref_jacobian.argtypes = [C.c_void_p, C.c_double, _D, _I, _I, _D, _D, C.c_long]
    lib.ref_integrate_stage.argtypes = [C.c_void_p, C.c_int, _D]
    lib.ref_field.argtypes = [C.c_int, C.c_long, _D, _D, _D]
    _libs[path] = lib
    return lib


def available(kind: str = "ref") -> bool:
    return os.path.exists(REF_LIB if kind == "ref" else PORT_LIB)


def params(cutoff_multiplier=1.0, prec=1e-8, step_size=1e-6, stress_kind=0,
           stress_value=0.0, stress_rate=0.0, spring_constant=1.0,
           pd_scaling=False, calculate_strain=False, order_parameter=False,
           max_step: Optional[float] = None) -> RefParams:
    return RefParams(float(cutoff_multiplier), float(prec), float(step_size), int(stress_kind),
                     float(stress_rate), float(spring_constant), float(stress_value),
                     int(bool(pd_scaling)), int(bool(calculate_strain)), int(bool(order_parameter)),
                     int(max_step is not None), float(max_step or 0.0))


SCALAR_NAMES = ["sim_time", "step_size", "successful_steps", "failed_steps", "energy",
                "strain", "max_error_ratio_sqr", "avg_speed", "vsquare", "energy_accum",
                "cutoff", "stress"]


class Sim:
    """One reference (or restatement) Simulation instance."""

    def __init__(self, xyb: np.ndarray, pd: Optional[np.ndarray], prm: RefParams, kind: str = "ref"):
        self.lib = _load(REF_LIB if kind == "ref" else PORT_LIB)
        self.xyb0 = np.ascontiguousarray(xyb, dtype=np.float64)
        self.n = self.xyb0.shape[0]
        self.pd = np.ascontiguousarray(pd if pd is not None else np.zeros((0, 2)), dtype=np.float64)
        self.p = self.pd.shape[0]
        self._pdbuf = self.pd.ctypes.data_as(C.c_void_p) if self.p else None
        self.h = self.lib.ref_create(self.n, self.xyb0.reshape(-1), self.p, self._pdbuf, C.byref(prm))

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self):
        out = np.zeros(8)
        self.lib.ref_get_params(self.h, out)
        return dict(zip(["cutoff", "cutoff_sqr", "one_per_cutoff_sqr", "A", "KASQR", "prec",
                         "step_size", "ic"], out))

    def step(self) -> bool:
        return bool(self.lib.ref_step(self.h))

    def scalars(self) -> dict:
        out = np.zeros(12)
        self.lib.ref_get_scalars(self.h, out)
        return dict(zip(SCALAR_NAMES, out))

    def config(self, which: int = 0) -> np.ndarray:
        out = np.zeros(self.n * 3)
        self.lib.ref_get_config(self.h, which, out)
        return out.reshape(self.n, 3)

    def vector(self, which: int) -> np.ndarray:
        out = np.zeros(self.n)
        self.lib.ref_get_vector(self.h, which, out)
        return out

    def set_state(self, xyb, step_size, sim_time=0.0, energy=0.0, strain=0.0, first_step=False):
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        self.lib.ref_set_state(self.h, a, float(step_size), float(sim_time), float(energy),
                               float(strain), int(first_step))

    def speeds(self, xyb, sim_time=0.0, stress_type=0):
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        v = np.zeros(self.n)
        tol = np.zeros(self.n)
        self.lib.ref_speeds(self.h, a, float(sim_time), int(stress_type), v, tol)
        return v, tol

    def jacobian(self, stepsize, xyb, cap: Optional[int] = None):
        """Returns (Ap, Ai, Ax, dvec) of the CSC Jacobian."""
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        cap = cap or max(1024, self.n * 64)
        while True:
            Ap = np.zeros(self.n + 1, dtype=np.int32)
            Ai = np.zeros(cap, dtype=np.int32)
            Ax = np.zeros(cap)
            d = np.zeros(self.n)
            nnz = self.lib.ref_jacobian(self.h, float(stepsize), a, Ap, Ai, Ax, d, cap)
            if nnz >= 0:
                return Ap, Ai[:nnz].copy(), Ax[:nnz].copy(), d
            cap = -nnz

    def integrate_stage(self, stage: int) -> np.ndarray:
        x = np.zeros(self.n)
        self.lib.ref_integrate_stage(self.h, int(stage), x)
        return x


def field(which: int, dx, dy, kind: str = "ref") -> np.ndarray:
    """which: 0 xy, 1 xy_diff_x, 2 xy_diff_x2 (AnalyticField.cpp:145-202)."""
    lib = _load(REF_LIB if kind == "ref" else PORT_LIB)
    dx = np.ascontiguousarray(dx, dtype=np.float64).reshape(-1)
    dy = np.ascontiguousarray(dy, dtype=np.float64).reshape(-1)
    out = np.zeros(dx.shape[0])
    lib.ref_field(int(which), dx.shape[0], dx, dy, out)
    return out


def csc_to_dense(Ap, Ai, Ax, n):
    A = np.zeros((n, n))
    for j in range(n):
        for p in range(Ap[j], Ap[j + 1]):
            A[Ai[p], j] += Ax[p]
    return A


# ------------------------------------------------------- eigenvalue analysis

def _ev_lib(kind: str):
    lib = _load(REF_LIB if kind == "ref" else PORT_LIB)
    if kind == "ref":
        if not hasattr(lib, "_ev_bound"):
            lib.ref_ev_decompose.argtypes = [C.c_int, _D, C.c_int, C.c_void_p, _D, _D, _D]
            lib._ev_bound = True
    elif not hasattr(lib, "_ev_bound"):
        lib.orc_ev_hessian.argtypes = [C.c_int, _D, C.c_int, C.c_void_p, _D]
        lib.orc_ev_deriv_literal.argtypes = [C.c_int, _D, _D, _D, C.c_double, _D]
        lib.orc_ev_correl_literal.argtypes = [C.c_int, _D, _D, C.c_int, _D]
        lib._ev_bound = True
    return lib


def _pd_arg(pd):
    pd = np.ascontiguousarray(pd if pd is not None else np.zeros((0, 2)), dtype=np.float64)
    return pd, (pd.ctypes.data_as(C.c_void_p) if pd.shape[0] else None)


def ev_decompose_ref(xyb, pd=None):
    """SpectralDecompositor::decompose of the reference compiled in place
    (src/spectral_decompositor.cpp:63-201) with the LAPACKE shim: (H, w, V),
    H the Hessian handed to LAPACKE_dsyevd, V[m] eigenvector m."""
    lib = _ev_lib("ref")
    a = np.ascontiguousarray(xyb, dtype=np.float64)
    n = a.shape[0]
    pd, pp = _pd_arg(pd)
    H, w, V = np.zeros(n * n), np.zeros(n), np.zeros(n * n)
    lib.ref_ev_decompose(n, a.reshape(-1), pd.shape[0], pp, H, w, V)
    return H.reshape(n, n), w, V.reshape(n, n)


def ev_hessian(xyb, pd=None) -> np.ndarray:
    """The restated Hessian (sdddst_oracle.c orc_ev_hessian), n x n."""
    lib = _ev_lib("port")
    a = np.ascontiguousarray(xyb, dtype=np.float64)
    n = a.shape[0]
    pd, pp = _pd_arg(pd)
    H = np.zeros(n * n)
    lib.orc_ev_hessian(n, a.reshape(-1), pd.shape[0], pp, H)
    return H.reshape(n, n)


def ev_analysis(xyb, pd, speeds, stress_derivative=1.0, nvec=10, deriv=False, corr_bins=0) -> dict:
    """The observables TimeSeriesProcessor::run writes for one configuration
    (src/time_series_processor.cpp:33-199): eigenvalues (ascending), the
    participation numbers 1/sum_j v_mj^4, the Burgers sums s_m = sum_j v_mj b_j
    and 1/Gael = s_m^2 / lambda_m, the first nvec eigenvectors, optionally the
    eigenvalue derivatives (literal n^4 loop) and the correlation matrices.
    The eigenpairs come from numpy.linalg.eigh (LAPACK's syevd driver, the
    one the reference calls)."""
    a = np.ascontiguousarray(xyb, dtype=np.float64)
    n = a.shape[0]
    H = ev_hessian(a, pd)
    w, Vc = np.linalg.eigh(H)
    V = np.ascontiguousarray(Vc.T)
    b = a[:, 2]
    s = V @ b
    out = dict(eigenvalues=w, participation=1.0 / np.sum(V ** 4, axis=1), burgers_sum=s, gan=s ** 2 / w,
               eigenvectors=V[:nvec].copy(), speeds=np.asarray(speeds, dtype=np.float64), hessian=H, V=V)
    lib = _ev_lib("port")
    if deriv:
        d = np.zeros(n)
        lib.orc_ev_deriv_literal(n, a.reshape(-1), V.reshape(-1), np.ascontiguousarray(out["speeds"]),
                                 float(stress_derivative), d)
        out["derivatives"] = d
    if corr_bins:
        cm = np.zeros(n * 3 * corr_bins * corr_bins)
        lib.orc_ev_correl_literal(n, a.reshape(-1), V.reshape(-1), int(corr_bins), cm)
        out["correlations"] = cm.reshape(n, 3, corr_bins, corr_bins)
    return out
