"""ctypes binding of the engine's C ABI (``include/sdddst_b200.h``).

This is the path tests and the bench call through: plain pointers and sizes,
no torch types.  Loading fails loudly when the CUDA library has not been
built; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsdddst_b200.so")

OK = 0
ERR_INVALID = -1
ERR_CUDA = -2
ERR_NOMEM = -3
ERR_SOLVER = -4
ERR_CAPACITY = -5
ERR_NONFINITE = -6

STRESS_ZERO, STRESS_FIXED_RATE, STRESS_SPRING, STRESS_CONSTANT = 0, 1, 2, 3
PAIRSUM_FP64, PAIRSUM_FP32 = 0, 1
FIELD_ANALYTIC, FIELD_TABULATED = 0, 1
SOLVER_GMRES, SOLVER_GMRES_JACOBI, SOLVER_GMRES_CLUSTER, SOLVER_DIRECT = 0, 1, 2, 3
SOLVER_GMRES_LEARNED, SOLVER_GMRES_NEUMANN, SOLVER_DIRECT_MIXED = 4, 5, 6

# Every extern "C" symbol of include/sdddst_b200.h.
EXPORTS = [
    "sdddst_default_params", "sdddst_ctx_create", "sdddst_ctx_destroy", "sdddst_last_error",
    "sdddst_set_state", "sdddst_get_scalars", "sdddst_get_config", "sdddst_get_vector",
    "sdddst_speeds", "sdddst_jacobian", "sdddst_solve", "sdddst_step", "sdddst_run",
    "sdddst_state_device", "sdddst_kernel_launches", "sdddst_upload_positions",
    "sdddst_download_positions", "sdddst_stream", "sdddst_vector_peaks", "sdddst_profile_pair_sum",
    "sdddst_speeds_noalloc", "sdddst_solver_stats", "sdddst_speeds_ext", "sdddst_set_scalars",
    "sdddst_update_params", "sdddst_solve_csc", "sdddst_batch_create", "sdddst_batch_destroy",
    "sdddst_batch_step", "sdddst_batch_get_scalars", "sdddst_batch_get_positions", "sdddst_batch_info",
    "sdddst_direct_stats", "sdddst_profile_direct", "sdddst_precond_apply", "sdddst_set_preconditioner_weights",
    "sdddst_learned_correction", "sdddst_solver_recoveries", "sdddst_batch_stats",
    "sdddst_batch_profile_pair_sum", "sdddst_ev_hessian", "sdddst_ev_analyze", "sdddst_ev_timings",
    "sdddst_learned_train_init", "sdddst_learned_train_step", "sdddst_learned_train_weights",
]


class Params(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("p", C.c_int),
        ("cutoff_multiplier", C.c_double), ("prec", C.c_double), ("step_size", C.c_double),
        ("A", C.c_double), ("KASQR", C.c_double), ("ic", C.c_int),
        ("stress_kind", C.c_int), ("stress_rate", C.c_double), ("spring_constant", C.c_double),
        ("stress_value", C.c_double), ("calculate_strain", C.c_int), ("max_step_limited", C.c_int),
        ("max_step", C.c_double), ("field", C.c_int), ("pairsum", C.c_int), ("solver", C.c_int),
        ("solver_tol", C.c_double), ("gmres_restart", C.c_int), ("max_iters", C.c_int),
        ("precond_theta", C.c_double), ("device", C.c_int), ("neumann_theta", C.c_double),
    ]


class EngineError(RuntimeError):
    def __init__(self, rc: int, msg: str):
        super().__init__(f"sdddst_b200 error {rc}: {msg}")
        self.rc = rc


_lib = None
_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_I = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def load(path: str = LIB_PATH):
    """Load the CUDA engine library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -m sdddst_b200.build`")
    lib = C.CDLL(path)
    lib.sdddst_default_params.argtypes = [C.POINTER(Params)]
    lib.sdddst_default_params.restype = None
    lib.sdddst_last_error.restype = C.c_char_p
    lib.sdddst_ctx_create.argtypes = [C.POINTER(Params), _D, C.c_void_p, C.POINTER(C.c_void_p)]
    lib.sdddst_ctx_destroy.argtypes = [C.c_void_p]
    lib.sdddst_set_state.argtypes = [C.c_void_p, _D, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
    lib.sdddst_get_scalars.argtypes = [C.c_void_p, _D]
    lib.sdddst_get_config.argtypes = [C.c_void_p, C.c_int, _D]
    lib.sdddst_get_vector.argtypes = [C.c_void_p, C.c_int, _D]
    lib.sdddst_speeds.argtypes = [C.c_void_p, _D, C.c_double, C.c_int, _D, _D]
    lib.sdddst_jacobian.argtypes = [C.c_void_p, C.c_double, _D, _I, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_long, C.POINTER(C.c_long)]
    lib.sdddst_solve.argtypes = [C.c_void_p, C.c_double, _D, _D, _D, C.POINTER(C.c_int)]
    lib.sdddst_step.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.sdddst_run.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.sdddst_state_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.sdddst_upload_positions.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.sdddst_download_positions.argtypes = [C.c_void_p, C.c_void_p]
    lib.sdddst_stream.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
    lib.sdddst_speeds_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                          C.c_void_p]
    lib.sdddst_speeds_ext.argtypes = [C.c_void_p, _D, C.c_double, _D, _D]
    lib.sdddst_set_scalars.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double]
    lib.sdddst_update_params.argtypes = [C.c_void_p, C.POINTER(Params)]
    lib.sdddst_solve_csc.argtypes = [C.c_void_p, _I, _I, _D, _D, _D, C.POINTER(C.c_int)]
    lib.sdddst_batch_create.argtypes = [C.POINTER(Params), C.c_int, _I, _D, C.POINTER(C.c_void_p)]
    lib.sdddst_batch_destroy.argtypes = [C.c_void_p]
    lib.sdddst_batch_step.argtypes = [C.c_void_p, _I]
    lib.sdddst_batch_get_scalars.argtypes = [C.c_void_p, _D]
    lib.sdddst_batch_get_positions.argtypes = [C.c_void_p, C.c_int, _D]
    lib.sdddst_batch_info.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_long), C.POINTER(C.c_long),
                                      C.POINTER(C.c_void_p)]
    lib.sdddst_solver_stats.argtypes = [C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_long)]
    lib.sdddst_batch_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_long)]
    lib.sdddst_batch_profile_pair_sum.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                                  C.POINTER(C.c_double)]
    lib.sdddst_solver_recoveries.argtypes = [C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_long),
                                             C.POINTER(C.c_long)]
    lib.sdddst_profile_pair_sum.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
    lib.sdddst_ev_hessian.argtypes = [C.c_void_p, _D, _D]
    lib.sdddst_ev_analyze.argtypes = [C.c_void_p, _D, C.c_double] + [C.c_void_p] * 6 + [C.c_int, C.c_void_p,
                                                                                        C.c_void_p, C.c_int]
    lib.sdddst_ev_timings.argtypes = [C.c_void_p, _D]
    _F = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
    lib.sdddst_learned_train_init.argtypes = [C.c_void_p, _F, C.c_long]
    lib.sdddst_learned_train_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_ulonglong, C.c_int,
                                              _D, C.c_void_p]
    lib.sdddst_learned_train_weights.argtypes = [C.c_void_p, _F, C.c_long]
    lib.sdddst_vector_peaks.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.sdddst_direct_stats.argtypes = [C.c_void_p, C.POINTER(C.c_long), C.POINTER(C.c_long),
                                        C.POINTER(C.c_double), C.POINTER(C.c_long), C.POINTER(C.c_int),
                                        C.POINTER(C.c_int)]
    lib.sdddst_profile_direct.argtypes = [C.c_void_p, C.c_double, C.c_int, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]
    lib.sdddst_precond_apply.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.sdddst_set_preconditioner_weights.argtypes = [C.c_void_p, C.c_void_p, C.c_long]
    lib.sdddst_learned_correction.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_long, C.POINTER(C.c_long)]
    lib.sdddst_kernel_launches.argtypes = [C.c_void_p]
    lib.sdddst_kernel_launches.restype = C.c_long
    _lib = lib
    return lib


def _check(rc: int):
    if rc != OK:
        raise EngineError(rc, load().sdddst_last_error().decode(errors="replace"))


def vector_peaks(device: int = 0):
    """Measured FP64 and FP32 FMA throughput (TFLOP/s) of the GPU."""
    a, b = C.c_double(0), C.c_double(0)
    _check(load().sdddst_vector_peaks(int(device), C.byref(a), C.byref(b)))
    return a.value, b.value


def default_params(**kw) -> Params:
    p = Params()
    load().sdddst_default_params(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def cli_params(n: int, cutoff_multiplier: float, prec: float, step_size: float = 1e-6, p: int = 0,
               pd_scaling: bool = False, **kw) -> Params:
    """Parameters as the reference CLI sets them (project_parser.cpp:137-298):
    SimulationData defaults, then step size, precision, cutoff multiplier and,
    when a point-defect file is given, A *= 1/sqrt(N) and KASQR *= N."""
    prm = default_params(n=n, p=p, cutoff_multiplier=cutoff_multiplier, prec=prec, step_size=step_size)
    if pd_scaling:
        prm.A = prm.A * (1.0 / np.sqrt(float(n)))
        prm.KASQR = prm.KASQR * float(n)
    for k, v in kw.items():
        setattr(prm, k, v)
    return prm


SCALAR_NAMES = ["sim_time", "step_size", "successful_steps", "failed_steps", "energy", "strain",
                "max_error_ratio_sqr", "avg_speed", "vsquare", "energy_accum", "cutoff", "stress"]


class Engine:
    """One device context (one simulated system on one GPU)."""

    def __init__(self, prm: Params, xyb: np.ndarray, pd: Optional[np.ndarray] = None):
        lib = load()
        self.lib = lib
        self.prm = prm
        xyb = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        self.n = prm.n
        if xyb.size != 3 * self.n:
            raise ValueError("xyb must hold n rows of (x, y, b)")
        self._pd = None
        pdp = None
        if prm.p > 0:
            self._pd = np.ascontiguousarray(pd, dtype=np.float64).reshape(-1)
            if self._pd.size != 2 * prm.p:
                raise ValueError("pd must hold p rows of (x, y)")
            pdp = self._pd.ctypes.data_as(C.c_void_p)
        h = C.c_void_p()
        _check(lib.sdddst_ctx_create(C.byref(prm), xyb, pdp, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.sdddst_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, xyb, step_size, sim_time=0.0, energy=0.0, strain=0.0, first_step=False):
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        _check(self.lib.sdddst_set_state(self.h, a, float(step_size), float(sim_time), float(energy),
                                         float(strain), int(first_step)))

    def scalars(self) -> dict:
        out = np.zeros(12)
        _check(self.lib.sdddst_get_scalars(self.h, out))
        return dict(zip(SCALAR_NAMES, out))

    def config(self, which: int = 0) -> np.ndarray:
        out = np.zeros(3 * self.n)
        _check(self.lib.sdddst_get_config(self.h, which, out))
        return out.reshape(self.n, 3)

    def vector(self, which: int) -> np.ndarray:
        out = np.zeros(self.n)
        _check(self.lib.sdddst_get_vector(self.h, which, out))
        return out

    def speeds(self, xyb, sim_time=0.0, stress_type=0):
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        v = np.zeros(self.n)
        tol = np.zeros(self.n)
        _check(self.lib.sdddst_speeds(self.h, a, float(sim_time), int(stress_type), v, tol))
        return v, tol

    def jacobian(self, h, xyb):
        """CSR of J: (row_ptr, col, val, dvec)."""
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        rp = np.zeros(self.n + 1, dtype=np.int32)
        nnz = C.c_long(0)
        rc = self.lib.sdddst_jacobian(self.h, float(h), a, rp, None, None, None, 0, C.byref(nnz))
        if rc not in (OK, ERR_CAPACITY):
            _check(rc)
        cap = nnz.value
        col = np.zeros(cap, dtype=np.int32)
        val = np.zeros(cap)
        d = np.zeros(self.n)
        _check(self.lib.sdddst_jacobian(self.h, float(h), a, rp, col.ctypes.data_as(C.c_void_p),
                                        val.ctypes.data_as(C.c_void_p), d.ctypes.data_as(C.c_void_p),
                                        cap, C.byref(nnz)))
        return rp, col[:nnz.value], val[:nnz.value], d

    def solve(self, h, xyb, rhs):
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        r = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros(self.n)
        it = C.c_int(0)
        _check(self.lib.sdddst_solve(self.h, float(h), a, r, x, C.byref(it)))
        return x, it.value

    def speeds_ext(self, xyb, tau_ext=0.0):
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        v = np.zeros(self.n)
        m = np.zeros(self.n)
        _check(self.lib.sdddst_speeds_ext(self.h, a, float(tau_ext), v, m))
        return v, m

    def solve_csc(self, Ap, Ai, Ax, b):
        x = np.zeros(self.n)
        it = C.c_int(0)
        _check(self.lib.sdddst_solve_csc(self.h, np.ascontiguousarray(Ap, dtype=np.int32),
                                         np.ascontiguousarray(Ai, dtype=np.int32),
                                         np.ascontiguousarray(Ax, dtype=np.float64),
                                         np.ascontiguousarray(b, dtype=np.float64), x, C.byref(it)))
        return x, it.value

    def step(self) -> bool:
        a = C.c_int(0)
        _check(self.lib.sdddst_step(self.h, C.byref(a)))
        return bool(a.value)

    def run(self, accepted_target: int, max_attempts: int):
        a, t = C.c_int(0), C.c_int(0)
        _check(self.lib.sdddst_run(self.h, int(accepted_target), int(max_attempts), C.byref(a), C.byref(t)))
        return a.value, t.value

    def upload_positions(self, x, recompute: bool = False):
        """x: a C-contiguous float64 array (pinned host memory is fastest)."""
        _check(self.lib.sdddst_upload_positions(self.h, C.c_void_p(x.ctypes.data if isinstance(x, np.ndarray)
                                                                    else int(x)), int(recompute)))

    def download_positions(self, x):
        _check(self.lib.sdddst_download_positions(self.h, C.c_void_p(x.ctypes.data if isinstance(x, np.ndarray)
                                                                      else int(x))))

    def stream(self) -> int:
        s = C.c_void_p()
        _check(self.lib.sdddst_stream(self.h, C.byref(s)))
        return s.value or 0

    def profile_pair_sum(self, reps: int = 3) -> float:
        """Mean device milliseconds of one pair-sum launch (CUDA events)."""
        ms = C.c_double(0)
        _check(self.lib.sdddst_profile_pair_sum(self.h, int(reps), C.byref(ms)))
        return ms.value

    def solver_stats(self):
        a, b = C.c_long(0), C.c_long(0)
        _check(self.lib.sdddst_solver_stats(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def solver_recoveries(self):
        """(preconditioner rebuilds, sparse-LU fallbacks, redone attempts)."""
        a, b, c = C.c_long(0), C.c_long(0), C.c_long(0)
        _check(self.lib.sdddst_solver_recoveries(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def learned_train_init(self, weights_fp32):
        """Starts training the learned correction from FP32 weights."""
        w = np.ascontiguousarray(weights_fp32, dtype=np.float32)
        _check(self.lib.sdddst_learned_train_init(self.h, w, w.size))

    def learned_train_step(self, h, probes=8, lr=1e-3, seed=0, apply=True, grad=False):
        """One training step on J(h) at the accepted configuration: returns
        (loss of B alone, loss of B + C[, gradient])."""
        from sdddst_b200.learned import weight_count
        loss = np.zeros(2)
        g = np.zeros(weight_count(), dtype=np.float32) if grad else None
        _check(self.lib.sdddst_learned_train_step(self.h, float(h), int(probes), float(lr), int(seed) & (2**64 - 1),
                                                  int(bool(apply)), loss,
                                                  g.ctypes.data_as(C.c_void_p) if grad else None))
        return (loss[0], loss[1], g) if grad else (loss[0], loss[1])

    def learned_train_weights(self) -> np.ndarray:
        from sdddst_b200.learned import weight_count
        w = np.zeros(weight_count(), dtype=np.float32)
        _check(self.lib.sdddst_learned_train_weights(self.h, w, w.size))
        return w

    def ev_hessian(self, xyb) -> np.ndarray:
        """The dense Hessian of SpectralDecompositor::decompose (n x n)."""
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        H = np.zeros(self.n * self.n)
        _check(self.lib.sdddst_ev_hessian(self.h, a, H))
        return H.reshape(self.n, self.n)

    def ev_analyze(self, xyb, sim_time=0.0, nvec=10, deriv=False, corr_bins=0) -> dict:
        """One configuration of the eigenvalue analysis (sdddst_ev_analyze):
        eigenvalues, participation, burgers_sum, gan, speeds, eigenvectors
        (nvec x n), derivatives (when deriv), correlations (n x 3 x S x S
        when corr_bins = S > 0)."""
        a = np.ascontiguousarray(xyb, dtype=np.float64).reshape(-1)
        n = self.n
        nv = min(int(nvec), n)
        out = {k: np.zeros(n) for k in ("eigenvalues", "participation", "burgers_sum", "gan", "speeds")}
        out["eigenvectors"] = np.zeros((nv, n))
        if deriv:
            out["derivatives"] = np.zeros(n)
        if corr_bins:
            out["correlations"] = np.zeros((n, 3, corr_bins, corr_bins))

        def ptr(k):
            return out[k].ctypes.data_as(C.c_void_p) if k in out else None
        _check(self.lib.sdddst_ev_analyze(self.h, a, float(sim_time), ptr("eigenvalues"), ptr("participation"),
                                          ptr("burgers_sum"), ptr("gan"), ptr("speeds"),
                                          out["eigenvectors"].ctypes.data_as(C.c_void_p) if nv else None, nv,
                                          ptr("derivatives"), ptr("correlations"), int(corr_bins)))
        return out

    def ev_timings(self) -> dict:
        ms = np.zeros(5)
        _check(self.lib.sdddst_ev_timings(self.h, ms))
        return dict(zip(["hessian", "eigensolver", "observables", "derivatives", "correlations"], ms))

    def update_params(self, **kw):
        """Changes mutable parameters of the live context (sdddst_update_params)."""
        for k, v in kw.items():
            if not hasattr(self.prm, k):
                raise AttributeError(k)
            setattr(self.prm, k, v)
        _check(self.lib.sdddst_update_params(self.h, C.byref(self.prm)))

    def direct_stats(self) -> dict:
        f, pp, fd = C.c_long(0), C.c_long(0), C.c_long(0)
        fl = C.c_double(0.0)
        nf, dp = C.c_int(0), C.c_int(0)
        _check(self.lib.sdddst_direct_stats(self.h, C.byref(f), C.byref(pp), C.byref(fl), C.byref(fd),
                                            C.byref(nf), C.byref(dp)))
        return {"factorizations": f.value, "perturbed_pivots": pp.value, "lu_flops": fl.value,
                "front_doubles": fd.value, "fronts": nf.value, "depth": dp.value}

    def profile_direct(self, h: float, reps: int = 2):
        """Mean device milliseconds of one sparse-LU factorization of J(h)
        at the accepted configuration and of one solve with it."""
        f, s = C.c_double(0.0), C.c_double(0.0)
        _check(self.lib.sdddst_profile_direct(self.h, float(h), int(reps), C.byref(f), C.byref(s)))
        return f.value, s.value

    def precond_apply(self, h: float, k: int, in_ptr: int, out_ptr: int, block_ptr: int = 0):
        """Cluster preconditioner of J(h) at the accepted configuration applied
        to k device vectors (raw device pointers, k x n doubles)."""
        _check(self.lib.sdddst_precond_apply(self.h, float(h), int(k), C.c_void_p(in_ptr), C.c_void_p(out_ptr),
                                             C.c_void_p(block_ptr) if block_ptr else None))

    def set_preconditioner_weights(self, bf16=None):
        """Loads the learned preconditioner's BF16 weights (uint16 bit
        patterns; default: the shipped sdddst_b200/learned_weights.npz)."""
        if bf16 is None:
            from sdddst_b200 import learned
            bf16 = learned.load_weights()
        w = np.ascontiguousarray(bf16, dtype=np.uint16)
        _check(self.lib.sdddst_set_preconditioner_weights(self.h, w.ctypes.data, int(w.size)))

    def learned_correction(self, h: float) -> np.ndarray:
        """Values of the learned correction C for J(h) at the accepted
        configuration, aligned with the CSR of jacobian()."""
        cap = C.c_long(0)
        probe = np.zeros(1, dtype=np.float32)
        rc = self.lib.sdddst_learned_correction(self.h, float(h), probe.ctypes.data, 0, C.byref(cap))
        if rc not in (OK, ERR_CAPACITY):
            _check(rc)
        out = np.zeros(max(1, cap.value), dtype=np.float32)
        _check(self.lib.sdddst_learned_correction(self.h, float(h), out.ctypes.data, out.size, C.byref(cap)))
        return out[:cap.value]

    def launches(self) -> int:
        return int(self.lib.sdddst_kernel_launches(self.h))


class Batch:
    """Independent systems of uneven size stepped together on one GPU."""

    def __init__(self, prm: Params, systems):
        lib = load()
        self.lib = lib
        self.sizes = np.array([len(s) for s in systems], dtype=np.int32)
        self.count = len(systems)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])
        xyb = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.float64) for s in systems]).reshape(-1))
        h = C.c_void_p()
        _check(lib.sdddst_batch_create(C.byref(prm), self.count, self.sizes, xyb, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.sdddst_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self) -> np.ndarray:
        acc = np.zeros(self.count, dtype=np.int32)
        _check(self.lib.sdddst_batch_step(self.h, acc))
        return acc.astype(bool)

    def scalars(self) -> np.ndarray:
        out = np.zeros(12 * self.count)
        _check(self.lib.sdddst_batch_get_scalars(self.h, out))
        return out.reshape(self.count, 12)

    def positions(self, which: int = 0):
        x = np.zeros(int(self.offsets[-1]))
        _check(self.lib.sdddst_batch_get_positions(self.h, which, x))
        return [x[self.offsets[k]:self.offsets[k + 1]] for k in range(self.count)]

    def stats(self):
        """{"graph": 1 when steps replay a captured CUDA graph, "redone": steps
        repeated host-driven after a failed deferred check}."""
        g, r = C.c_int(0), C.c_long(0)
        _check(self.lib.sdddst_batch_stats(self.h, C.byref(g), C.byref(r)))
        return {"graph": g.value, "redone": r.value}

    def profile_pair_sum(self, reps: int = 3):
        """(mean device ms of one pair-sum launch over all systems, unique pairs)."""
        ms, pairs = C.c_double(0), C.c_double(0)
        _check(self.lib.sdddst_batch_profile_pair_sum(self.h, int(reps), C.byref(ms), C.byref(pairs)))
        return ms.value, pairs.value

    def info(self):
        t, n, l, s = C.c_int(0), C.c_long(0), C.c_long(0), C.c_void_p()
        _check(self.lib.sdddst_batch_info(self.h, C.byref(t), C.byref(n), C.byref(l), C.byref(s)))
        return {"tile": t.value, "total": n.value, "launches": l.value, "stream": s.value or 0}
