"""B200 PDLP engine -- Python mirror of the reference solver's GPU PDLP entry point.

The product is ``libb200pdlp.so`` (CUDA sm_100a kernels + C++ host side + the C
ABI declared in ``include/b200_pdlp.h``). This module binds that ABI with
ctypes and mirrors the reference interface it replaces:

* ``solve_pdhg_gpu(unscaled_form, scaled_form, Dr, Dc, eta, max_iterations,
  check_every, tol, stop_flag)`` -> ``PdlpResult``: the same arguments, in the same
  order and with the same meaning, as ``solve_pdhg_gpu`` in the reference's
  include/pdlp_gpu.hpp:22-25; ``PdlpResult`` has the fields of
  include/pdlp.hpp:18-24. Errors raise ``RuntimeError`` (the reference throws
  ``std::runtime_error``, gpu/pdlp_gpu_solve.cu:32-38); a non-converged solve is
  a normal result with ``converged = False``.
* ``RangedLP`` holds an LP as include/ranged_lp.hpp:10-27 does (COO matrix).
* ``Engine`` keeps a problem resident on the GPU for repeated solves.

There is no CPU fallback: importing works without a GPU, but every solve
needs the CUDA library and a device, and fails loudly otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb200pdlp.so")
INCLUDE_H = os.path.join(os.path.dirname(HERE), "include", "b200_pdlp.h")

B2_OK, B2_ERR_INVALID, B2_ERR_CUDA, B2_ERR_OOM, B2_ERR_TIMEOUT, B2_ERR_NO_DEVICE, B2_ERR_NONFINITE, \
    B2_ERR_UNSUPPORTED, B2_ERR_PENDING, B2_ERR_INFEASIBLE, B2_ERR_UNBOUNDED = range(11)
PREC_FP64, PREC_MIXED = 0, 1
EXIT_CONVERGED, EXIT_MAX_ITER, EXIT_STOPPED, EXIT_TIME_LIMIT = 1, 2, 3, 4

EXPORTED = [
    "b2_default_opts", "b2_solve_pdhg_gpu", "b2_solve_pdhg_gpu_ex", "b2_solve_pdhg_gpu_noalloc",
    "b2_engine_create", "b2_engine_solve",
    "b2_engine_destroy", "b2_engine_get_info", "b2_engine_spmv", "b2_engine_spmv_bench", "b2_engine_trace",
    "b2_batch_create", "b2_batch_solve", "b2_batch_get_solution", "b2_batch_get_info", "b2_batch_spmv",
    "b2_batch_destroy", "b2_shape_class", "b2_default_tune_table", "b2_batch_autotune",
    "b2_server_create", "b2_server_submit", "b2_server_submit_file", "b2_server_submit_lp", "b2_server_wait",
    "b2_server_stats_get", "b2_pdlp_form_build", "b2_pdlp_form_view", "b2_pdlp_form_extract",
    "b2_pdlp_form_destroy", "b2_presolve", "b2_presolved_view", "b2_postsolve", "b2_presolved_destroy",
    "b2_server_destroy", "b2_lp_write", "b2_lp_read_dims", "b2_lp_read",
    "b2_layout_digest", "b2_layout_get_stats", "b2_request_work", "b2_request_cost", "b2_shard_plan", "b2_pool_create", "b2_pool_submit", "b2_pool_submit_file",
    "b2_pool_wait", "b2_pool_stats_get", "b2_pool_destroy",
    "b2_scale", "b2_scale_gpu",
    "b2_gen_random_lp", "b2_gen_transport", "b2_last_error", "b2_version",
]


class B2Error(RuntimeError):
    """A non-zero B2_ERR_* status from the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"b200 pdlp error {code}: {msg}")
        self.code = code


class _LPView(C.Structure):
    _fields_ = [("m", C.c_int32), ("n", C.c_int32), ("nnz", C.c_int64),
                ("row_idx", C.c_void_p), ("col_idx", C.c_void_p), ("val", C.c_void_p),
                ("c", C.c_void_p), ("rL", C.c_void_p), ("rU", C.c_void_p),
                ("l", C.c_void_p), ("u", C.c_void_p), ("obj_offset", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("check_every", C.c_int32), ("tol", C.c_double),
                ("precision", C.c_int32), ("switch_tol", C.c_double), ("stall_checks", C.c_int32),
                ("time_limit_s", C.c_double), ("barrier_timeout_s", C.c_double), ("max_ctas", C.c_int32),
                ("lane_target", C.c_int32), ("sigma_window", C.c_int32), ("return_current", C.c_int32),
                ("stream", C.c_void_p), ("debug_delay_us", C.c_int32), ("batch_cluster_nnz", C.c_int32),
                ("batch_block", C.c_int32), ("stop_poll", C.c_void_p), ("stop_ctx", C.c_void_p),
                ("tune", C.c_void_p), ("batch_tail_attempts", C.c_int32), ("long_rows", C.c_int32)]


TUNE_CLASSES = 20


class TuneTable(C.Structure):
    """Lane target per shape class (b2_tune_table)."""
    _fields_ = [("lane_target", C.c_int32 * TUNE_CLASSES), ("us_per_attempt", C.c_double * TUNE_CLASSES)]


class _Result(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("restarts", C.c_int32), ("converged", C.c_int32),
                ("accepted", C.c_int32), ("eps_P", C.c_double), ("eps_D", C.c_double), ("eps_G", C.c_double),
                ("objective", C.c_double), ("exit_reason", C.c_int32), ("checks", C.c_int32),
                ("fp32_attempts", C.c_int32), ("fp32_accepted", C.c_int32), ("device_ms", C.c_double),
                ("host_ms", C.c_double), ("final_eta", C.c_double), ("final_omega", C.c_double),
                ("group_ctas", C.c_int32)]


class BatchInfo(C.Structure):
    _fields_ = [("n_lp", C.c_int32), ("sum_m", C.c_int64), ("sum_n", C.c_int64), ("sum_nnz", C.c_int64),
                ("sum_padded", C.c_int64), ("max_ctas", C.c_int32), ("threads_per_cta", C.c_int32),
                ("device_bytes", C.c_int64), ("last_launch_ctas", C.c_int32)]


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_double), ("round_ms", C.c_double), ("max_resident", C.c_int32),
                ("prep_threads", C.c_int32), ("grid_nnz", C.c_int64), ("grid_slice_ms", C.c_double),
                ("cluster_nnz", C.c_int64), ("gpu_scale_nnz", C.c_int64)]


class RequestInfo(C.Structure):
    _fields_ = [("submit_s", C.c_double), ("admit_s", C.c_double), ("done_s", C.c_double),
                ("prep_ms", C.c_double), ("rounds", C.c_int32), ("lane", C.c_int32), ("device_bytes", C.c_int64),
                ("form_eps", C.c_double * 3), ("presolved_m", C.c_int32), ("presolved_n", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("rounds", C.c_int64), ("grid_slices", C.c_int64), ("resident", C.c_int32),
                ("queued", C.c_int32), ("bytes_in_use", C.c_int64), ("peak_bytes", C.c_int64),
                ("busy_ms", C.c_double), ("backlog_work", C.c_int64)]


class EngineInfo(C.Structure):
    _fields_ = [("m", C.c_int32), ("n", C.c_int32), ("nnz", C.c_int64), ("a_slices", C.c_int64),
                ("at_slices", C.c_int64), ("a_padded", C.c_int64), ("at_padded", C.c_int64),
                ("values_exact_fp32", C.c_int32), ("ctas", C.c_int32), ("threads_per_cta", C.c_int32),
                ("sm_count", C.c_int32), ("device_bytes", C.c_int64)]


class LayoutStats(C.Structure):
    _fields_ = [("a_slices", C.c_int64), ("at_slices", C.c_int64), ("a_padded", C.c_int64),
                ("at_padded", C.c_int64), ("a_groups", C.c_int64), ("at_groups", C.c_int64),
                ("a_dense", C.c_int64), ("at_dense", C.c_int64)]


_lib = None
_lib_lock = threading.Lock()


def lib():
    """The loaded CUDA library; raises if it has not been built."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"libb200pdlp.so is not built ({LIB_PATH}); run __graft_entry__.build()")
            L = C.CDLL(LIB_PATH)
            vp, i32, i64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
            L.b2_last_error.restype = C.c_char_p
            L.b2_version.restype = C.c_char_p
            L.b2_default_opts.argtypes = [C.POINTER(SolveOpts)]
            L.b2_solve_pdhg_gpu.argtypes = [C.POINTER(_LPView), C.POINTER(_LPView), vp, vp, f64, i32, i32, f64,
                                            vp, vp, vp, C.POINTER(_Result)]
            L.b2_solve_pdhg_gpu_ex.argtypes = [C.POINTER(_LPView), C.POINTER(_LPView), vp, vp,
                                               C.POINTER(SolveOpts), vp, vp, vp, C.POINTER(_Result)]
            L.b2_solve_pdhg_gpu_noalloc.argtypes = [C.POINTER(_LPView), C.POINTER(_LPView), vp, vp,
                                                    C.POINTER(SolveOpts), vp, vp, C.POINTER(_Result)]
            L.b2_engine_create.argtypes = [C.POINTER(_LPView), C.POINTER(_LPView), vp, vp, C.POINTER(SolveOpts),
                                           C.POINTER(vp)]
            L.b2_engine_solve.argtypes = [vp, C.POINTER(SolveOpts), vp, vp, vp, C.POINTER(_Result)]
            L.b2_engine_destroy.argtypes = [vp]
            L.b2_engine_destroy.restype = None
            L.b2_engine_get_info.argtypes = [vp, C.POINTER(EngineInfo)]
            L.b2_engine_spmv.argtypes = [vp, i32, vp, vp]
            L.b2_engine_spmv_bench.argtypes = [vp, i32, i32, i32, vp, C.POINTER(f64)]
            L.b2_engine_trace.argtypes = [vp, vp, i32, C.POINTER(i32)]
            L.b2_batch_create.argtypes = [i32, C.POINTER(_LPView), C.POINTER(_LPView), C.POINTER(vp), C.POINTER(vp),
                                          C.POINTER(SolveOpts), C.POINTER(vp)]
            L.b2_batch_solve.argtypes = [vp, C.POINTER(SolveOpts), vp, C.POINTER(_Result), C.POINTER(f64)]
            L.b2_batch_get_solution.argtypes = [vp, i32, vp, vp]
            L.b2_batch_get_info.argtypes = [vp, C.POINTER(BatchInfo)]
            L.b2_batch_spmv.argtypes = [vp, i32, i32, vp, vp]
            L.b2_batch_destroy.argtypes = [vp]
            L.b2_shape_class.argtypes = [i32, i32, i64]
            L.b2_shape_class.restype = i32
            L.b2_default_tune_table.argtypes = [C.POINTER(TuneTable)]
            L.b2_default_tune_table.restype = None
            L.b2_batch_autotune.argtypes = [i32, C.POINTER(_LPView), C.POINTER(_LPView), C.POINTER(vp), C.POINTER(vp),
                                            C.POINTER(SolveOpts), C.POINTER(TuneTable)]
            L.b2_batch_destroy.restype = None
            L.b2_server_create.argtypes = [C.POINTER(ServerOpts), C.POINTER(SolveOpts), C.POINTER(vp)]
            L.b2_server_submit.argtypes = [vp, C.POINTER(_LPView), C.POINTER(i64)]
            L.b2_server_submit_file.argtypes = [vp, C.c_char_p, C.POINTER(i64)]
            L.b2_server_submit_lp.argtypes = [vp, C.POINTER(_LPView), i32, C.POINTER(i64)]
            L.b2_pdlp_form_build.argtypes = [C.POINTER(_LPView), C.POINTER(vp)]
            L.b2_pdlp_form_view.argtypes = [vp, C.POINTER(_LPView)]
            L.b2_pdlp_form_view.restype = None
            L.b2_pdlp_form_extract.argtypes = [vp, vp, vp, vp, vp]
            L.b2_pdlp_form_destroy.argtypes = [vp]
            L.b2_pdlp_form_destroy.restype = None
            L.b2_presolve.argtypes = [C.POINTER(_LPView), C.POINTER(vp), C.POINTER(i32)]
            L.b2_presolved_view.argtypes = [vp, C.POINTER(_LPView)]
            L.b2_presolved_view.restype = None
            L.b2_postsolve.argtypes = [vp, vp, vp, vp, vp]
            L.b2_presolved_destroy.argtypes = [vp]
            L.b2_presolved_destroy.restype = None
            L.b2_lp_write.argtypes = [C.c_char_p, C.POINTER(_LPView)]
            L.b2_lp_read_dims.argtypes = [C.c_char_p, C.POINTER(i32), C.POINTER(i32), C.POINTER(i64)]
            L.b2_lp_read.argtypes = [C.c_char_p] + [vp] * 8 + [C.POINTER(f64)]
            L.b2_server_wait.argtypes = [vp, i64, f64, vp, vp, C.POINTER(_Result), C.POINTER(RequestInfo)]
            L.b2_server_stats_get.argtypes = [vp, C.POINTER(ServerStats)]
            L.b2_server_destroy.argtypes = [vp]
            L.b2_layout_get_stats.argtypes = [C.POINTER(_LPView), C.POINTER(_LPView), vp, vp, i32,
                                              C.POINTER(LayoutStats)]
            L.b2_layout_digest.argtypes = [C.POINTER(_LPView), C.POINTER(_LPView), vp, vp, i32, i32,
                                           C.POINTER(C.c_uint64)]
            L.b2_request_work.argtypes = [i32, i32, i64]
            L.b2_request_work.restype = i64
            L.b2_request_cost.argtypes = [i32, i32, i64]
            L.b2_request_cost.restype = i64
            L.b2_shard_plan.argtypes = [vp, i64, i32, i32, vp]
            L.b2_pool_create.argtypes = [vp, i32, C.POINTER(ServerOpts), C.POINTER(SolveOpts), C.POINTER(vp)]
            L.b2_pool_submit.argtypes = [vp, C.POINTER(_LPView), C.POINTER(i64)]
            L.b2_pool_submit_file.argtypes = [vp, C.c_char_p, C.POINTER(i64)]
            L.b2_pool_wait.argtypes = [vp, i64, f64, vp, vp, C.POINTER(_Result), C.POINTER(RequestInfo),
                                       C.POINTER(i32)]
            L.b2_pool_stats_get.argtypes = [vp, i32, C.POINTER(ServerStats)]
            L.b2_pool_destroy.argtypes = [vp]
            L.b2_server_destroy.restype = None
            L.b2_scale.argtypes = [C.POINTER(_LPView), i32] + [vp] * 8
            L.b2_scale_gpu.argtypes = [C.POINTER(_LPView), i32] + [vp] * 8
            L.b2_gen_random_lp.argtypes = [i32, i32, i32, C.c_uint64, i32] + [vp] * 8
            L.b2_gen_transport.argtypes = [i32, i32, C.c_uint64] + [vp] * 8
            _lib = L
        return _lib


def _check(rc: int):
    if rc != B2_OK:
        raise B2Error(rc, lib().b2_last_error().decode())


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


@dataclass
class RangedLP:
    """rL <= A x <= rU, l <= x <= u, min c'x + obj_offset (include/ranged_lp.hpp:10-27), A in COO."""

    m: int
    n: int
    row: np.ndarray
    col: np.ndarray
    val: np.ndarray
    c: np.ndarray
    rL: np.ndarray
    rU: np.ndarray
    l: np.ndarray
    u: np.ndarray
    obj_offset: float = 0.0

    def __post_init__(self):
        self.m, self.n = int(self.m), int(self.n)
        self.row = np.ascontiguousarray(self.row, np.int32)
        self.col = np.ascontiguousarray(self.col, np.int32)
        for k in ("val", "c", "rL", "rU", "l", "u"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), np.float64))
        self.obj_offset = float(self.obj_offset)

    @property
    def nnz(self) -> int:
        return int(self.val.size)

    @classmethod
    def like(cls, other) -> "RangedLP":
        """Copy of any object with the same fields (e.g. the oracle's LPForm)."""
        return cls(other.m, other.n, other.row, other.col, other.val, other.c, other.rL, other.rU, other.l,
                   other.u, getattr(other, "obj_offset", 0.0))

    def view(self) -> _LPView:
        return _LPView(self.m, self.n, self.nnz, _ptr(self.row), _ptr(self.col), _ptr(self.val), _ptr(self.c),
                       _ptr(self.rL), _ptr(self.rU), _ptr(self.l), _ptr(self.u), self.obj_offset)


@dataclass
class PdlpResult:
    """Fields of the reference's PdlpResult (include/pdlp.hpp:18-24) plus engine counters."""

    x: np.ndarray
    y: np.ndarray
    iterations: int = 0
    converged: bool = False
    eps_P: float = 0.0
    eps_D: float = 0.0
    eps_G: float = 0.0
    restarts: int = 0
    stats: dict = field(default_factory=dict)


class StopFlag:
    """Cooperative cancellation word, the counterpart of std::atomic<bool>* stop_flag
    (include/pdlp.hpp:30-34): set() from any thread; the device polls it."""

    def __init__(self):
        self._v = C.c_int32(0)

    def set(self):
        self._v.value = 1

    def clear(self):
        self._v.value = 0

    def is_set(self) -> bool:
        return bool(self._v.value)

    @property
    def ptr(self):
        return C.addressof(self._v)


def default_opts(**kw) -> SolveOpts:
    o = SolveOpts()
    lib().b2_default_opts(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        if k == "tune" and isinstance(v, TuneTable):
            v = C.addressof(v)  # the caller keeps the table alive while these options are in use
        setattr(o, k, v)
    return o


def _result(r: _Result, x, y) -> PdlpResult:
    stats = {k: getattr(r, k) for k, _ in _Result._fields_}
    return PdlpResult(x=x, y=y, iterations=r.iterations, converged=bool(r.converged), eps_P=r.eps_P,
                      eps_D=r.eps_D, eps_G=r.eps_G, restarts=r.restarts, stats=stats)


def _vec(a, n) -> np.ndarray:
    a = np.ascontiguousarray(a, np.float64)
    if a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def solve_pdhg_gpu(unscaled_form: RangedLP, scaled_form: RangedLP, Dr, Dc, eta: float = 0.99,
                   max_iterations: int = 200000, check_every: int = 64, tol: float = 1e-6,
                   stop_flag: Optional[StopFlag] = None, **opts) -> PdlpResult:
    """Drop-in for the reference's solve_pdhg_gpu (include/pdlp_gpu.hpp:22-25).

    unscaled_form is the PDLP form (build_pdlp_form), scaled_form = scale(unscaled_form)
    with scalings Dr, Dc. `eta` is ignored: the step size is adaptive, as in the
    reference (gpu/pdlp_gpu_solve.cu:263). Extra keyword options map to
    ``b2_solve_opts`` (precision, switch_tol, time_limit_s, ...).
    """
    U = RangedLP.like(unscaled_form)
    S = RangedLP.like(scaled_form)
    Dr = _vec(Dr, U.m)
    Dc = _vec(Dc, U.n)
    o = default_opts(max_iterations=int(max_iterations), check_every=int(check_every), tol=float(tol), **opts)
    x = np.zeros(max(U.n, 1))
    y = np.zeros(max(U.m, 1))
    r = _Result()
    uv, sv = U.view(), S.view()
    _check(lib().b2_solve_pdhg_gpu_ex(C.byref(uv), C.byref(sv), _ptr(Dr), _ptr(Dc), C.byref(o),
                                      stop_flag.ptr if stop_flag else None, _ptr(x), _ptr(y), C.byref(r)))
    return _result(r, x[:U.n], y[:U.m])


class Engine:
    """A PDLP problem resident in HBM (b2_engine_*): create once, solve many times."""

    def __init__(self, unscaled_form: RangedLP, scaled_form: RangedLP, Dr, Dc, **opts):
        self.U = RangedLP.like(unscaled_form)
        S = RangedLP.like(scaled_form)
        Dr = _vec(Dr, self.U.m)
        Dc = _vec(Dc, self.U.n)
        o = default_opts(**opts)
        h = C.c_void_p()
        uv, sv = self.U.view(), S.view()
        _check(lib().b2_engine_create(C.byref(uv), C.byref(sv), _ptr(Dr), _ptr(Dc), C.byref(o), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().b2_engine_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def solve(self, max_iterations: int = 200000, check_every: int = 64, tol: float = 1e-6,
              stop_flag: Optional[StopFlag] = None, copy_out: bool = True, **opts) -> PdlpResult:
        o = default_opts(max_iterations=int(max_iterations), check_every=int(check_every), tol=float(tol), **opts)
        x = np.zeros(max(self.U.n, 1)) if copy_out else None
        y = np.zeros(max(self.U.m, 1)) if copy_out else None
        r = _Result()
        _check(lib().b2_engine_solve(self._h, C.byref(o), stop_flag.ptr if stop_flag else None, _ptr(x), _ptr(y),
                                     C.byref(r)))
        return _result(r, None if x is None else x[:self.U.n], None if y is None else y[:self.U.m])

    def info(self) -> dict:
        i = EngineInfo()
        _check(lib().b2_engine_get_info(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in EngineInfo._fields_}

    def spmv(self, which: int, x) -> np.ndarray:
        """A x (which=0) or A^T x (which=1) through the device SpMV (FP64 accumulation)."""
        rows, cols = (self.U.m, self.U.n) if which == 0 else (self.U.n, self.U.m)
        xx = _vec(x, cols)
        if xx.size == 0:
            xx = np.zeros(1)
        y = np.zeros(max(rows, 1))
        _check(lib().b2_engine_spmv(self._h, which, _ptr(xx), _ptr(y)))
        return y[:rows]

    TRACE_FIELDS = ("attempts", "accepted", "eps_P", "eps_D", "eps_G", "avg_eps_P", "avg_eps_D", "avg_eps_G",
                    "omega", "eta", "flags", "avg_weight")

    def trace(self, max_records: int = 65536) -> np.ndarray:
        """Per-check records of the last solve, shape (checks, 12), columns TRACE_FIELDS."""
        out = np.zeros((max_records, len(self.TRACE_FIELDS)))
        n = C.c_int32()
        _check(lib().b2_engine_trace(self._h, _ptr(out), max_records, C.byref(n)))
        return out[:n.value]

    def spmv_bench(self, which: int, precision: int = PREC_MIXED, reps: int = 20, stream=None) -> float:
        ms = C.c_double()
        _check(lib().b2_engine_spmv_bench(self._h, which, precision, reps, stream, C.byref(ms)))
        return ms.value


class Batch:
    """Many LPs in one persistent launch (b2_batch_*): one CTA per LP, a device
    work queue, retired LPs hand their CTA to the next. problems is a list of
    (unscaled_form, scaled_form, Dr, Dc) tuples, each exactly what
    solve_pdhg_gpu takes; LP i's answer equals solve_pdhg_gpu on LP i."""

    def __init__(self, problems, **opts):
        self.n = len(problems)
        self._keep = []
        U_arr = (_LPView * self.n)()
        S_arr = (_LPView * self.n)()
        dr_arr = (C.c_void_p * self.n)()
        dc_arr = (C.c_void_p * self.n)()
        self.dims = []
        for i, (U, S, Dr, Dc) in enumerate(problems):
            U = RangedLP.like(U)
            S = RangedLP.like(S)
            Dr = _vec(Dr, U.m)
            Dc = _vec(Dc, U.n)
            if Dr.size == 0:
                Dr = np.zeros(1)
            if Dc.size == 0:
                Dc = np.zeros(1)
            self._keep += [U, S, Dr, Dc]
            U_arr[i] = U.view()
            S_arr[i] = S.view()
            dr_arr[i] = _ptr(Dr)
            dc_arr[i] = _ptr(Dc)
            self.dims.append((U.m, U.n))
        o = default_opts(**opts)
        h = C.c_void_p()
        _check(lib().b2_batch_create(self.n, U_arr, S_arr, dr_arr, dc_arr, C.byref(o), C.byref(h)))
        self._h = h
        self._keep = []  # the engine holds its own copy of the data

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().b2_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def solve(self, max_iterations: int = 200000, check_every: int = 64, tol: float = 1e-6,
              stop_flag: Optional[StopFlag] = None, **opts):
        """Returns (list of per-LP stats dicts, total device ms of the launch)."""
        o = default_opts(max_iterations=int(max_iterations), check_every=int(check_every), tol=float(tol), **opts)
        res = (_Result * self.n)()
        ms = C.c_double()
        _check(lib().b2_batch_solve(self._h, C.byref(o), stop_flag.ptr if stop_flag else None, res, C.byref(ms)))
        out = []
        for r in res:
            d = {k: getattr(r, k) for k, _ in _Result._fields_}
            d["converged"] = bool(d["converged"])
            out.append(d)
        return out, ms.value

    def solution(self, i: int):
        m, n = self.dims[i]
        x = np.zeros(max(n, 1))
        y = np.zeros(max(m, 1))
        _check(lib().b2_batch_get_solution(self._h, i, _ptr(x), _ptr(y)))
        return x[:n], y[:m]

    def spmv(self, i: int, which: int, x) -> np.ndarray:
        """A x (which=0) or A^T x (which=1) of LP i through the packed device layout."""
        m, n = self.dims[i]
        rows, cols = (m, n) if which == 0 else (n, m)
        xx = _vec(x, cols)
        if xx.size == 0:
            xx = np.zeros(1)
        y = np.zeros(max(rows, 1))
        _check(lib().b2_batch_spmv(self._h, i, which, _ptr(xx), _ptr(y)))
        return y[:rows]

    def info(self) -> dict:
        i = BatchInfo()
        _check(lib().b2_batch_get_info(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in BatchInfo._fields_}


class Server:
    """The served stream (b2_server_*): submit LPs in unscaled PDLP form as they
    arrive; the server scales and lays them out on its own threads, admits
    them under an HBM budget and solves them by continuous batching (rounds
    of the batched kernel; LPs keep their state on the device between
    rounds). wait(ticket) returns (PdlpResult, info dict)."""

    def __init__(self, hbm_budget_bytes: float = 0.0, round_ms: float = 0.0, max_resident: int = 0,
                 prep_threads: int = 0, grid_nnz: int = 0, grid_slice_ms: float = 0.0, cluster_nnz: int = 0,
                 gpu_scale_nnz: int = 0, **opts):
        so = ServerOpts(float(hbm_budget_bytes), float(round_ms), int(max_resident), int(prep_threads),
                        int(grid_nnz), float(grid_slice_ms), int(cluster_nnz), int(gpu_scale_nnz))
        o = default_opts(**opts)
        h = C.c_void_p()
        _check(lib().b2_server_create(C.byref(so), C.byref(o), C.byref(h)))
        self._h = h
        self._dims = {}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().b2_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, unscaled_form: RangedLP) -> int:
        U = RangedLP.like(unscaled_form)
        t = C.c_int64()
        _check(lib().b2_server_submit(self._h, C.byref(U.view()), C.byref(t)))
        self._dims[t.value] = (U.m, U.n)
        return t.value

    def submit_lp(self, lp: RangedLP, presolve: bool = True) -> int:
        """Submits an LP as the caller has it (b2_server_submit_lp): presolved,
        put in PDLP form and scaled on the server's threads; wait() returns the
        original LP's point (postsolved) with verify()'s figures on it."""
        L = RangedLP.like(lp)
        t = C.c_int64()
        _check(lib().b2_server_submit_lp(self._h, C.byref(L.view()), int(bool(presolve)), C.byref(t)))
        self._dims[t.value] = (L.m, L.n)
        return t.value

    def submit_file(self, path: str) -> int:
        """Submits an LP stored with write_lp; the server reads it on its own threads."""
        m, n, _ = lp_file_dims(path)
        t = C.c_int64()
        _check(lib().b2_server_submit_file(self._h, os.fsencode(path), C.byref(t)))
        self._dims[t.value] = (m, n)
        return t.value

    def wait(self, ticket: int, timeout_s: float = -1.0):
        """(PdlpResult, info) once the ticket is done; None if timeout_s passed first."""
        m, n = self._dims[ticket]
        x = np.zeros(max(n, 1))
        y = np.zeros(max(m, 1))
        r = _Result()
        inf = RequestInfo()
        rc = lib().b2_server_wait(self._h, int(ticket), float(timeout_s), _ptr(x), _ptr(y), C.byref(r), C.byref(inf))
        if rc == B2_ERR_PENDING:
            return None
        del self._dims[ticket]
        _check(rc)
        info = {k: getattr(inf, k) for k, _ in RequestInfo._fields_}
        info["form_eps"] = list(inf.form_eps)
        return _result(r, x[:n], y[:m]), info

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().b2_server_stats_get(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}


def layout_digest(unscaled_form: RangedLP, scaled_form: RangedLP, Dr, Dc, threads: int = 1,
                  whole_gpu: bool = True) -> int:
    """64-bit digest of the device layout built on the host with `threads`
    threads (b2_layout_digest): the one-LP engine's (whole_gpu) or a batched
    LP's. Needs no GPU."""
    U = RangedLP.like(unscaled_form)
    S = RangedLP.like(scaled_form)
    dr = _vec(Dr, U.m)
    dc = _vec(Dc, U.n)
    d = C.c_uint64()
    _check(lib().b2_layout_digest(C.byref(U.view()), C.byref(S.view()), _ptr(dr), _ptr(dc), int(threads),
                                  int(bool(whole_gpu)), C.byref(d)))
    return d.value


def layout_stats(unscaled_form: RangedLP, scaled_form: RangedLP, Dr, Dc, whole_gpu: bool = True) -> dict:
    """Shape of the device layout (b2_layout_get_stats; no GPU): slice
    records, stored entries, split groups and dense-run records of A and A^T."""
    U = RangedLP.like(unscaled_form)
    S = RangedLP.like(scaled_form)
    dr = _vec(Dr, U.m)
    dc = _vec(Dc, U.n)
    st = LayoutStats()
    _check(lib().b2_layout_get_stats(C.byref(U.view()), C.byref(S.view()), _ptr(dr), _ptr(dc),
                                     int(bool(whole_gpu)), C.byref(st)))
    return {k: getattr(st, k) for k, _ in LayoutStats._fields_}


# --------------------------------------------------- shares over several GPUs
def request_work(m: int, n: int, nnz: int) -> int:
    """The load unit of sharding and routing: 2 nnz + m + n (b2_request_work)."""
    return int(lib().b2_request_work(int(m), int(n), int(nnz)))


def request_cost(m: int, n: int, nnz: int) -> int:
    """Expected cost of a whole solve: request_work x round(167 m^0.657)
    attempts (b2_request_cost), the load of batch and stream shares."""
    return int(lib().b2_request_cost(int(m), int(n), int(nnz)))


def shard_plan(work, parts: int, online: bool = False) -> np.ndarray:
    """Share index of every item (b2_shard_plan): online=False, longest load
    first to the least-loaded share (a batch); online=True, in the given order
    to the least-loaded share so far (a stream). Every rank computes the same
    plan from the same list, so no collective is needed."""
    w = np.ascontiguousarray(work, dtype=np.int64)
    out = np.zeros(max(w.size, 1), np.int32)
    _check(lib().b2_shard_plan(_ptr(w), int(w.size), int(parts), int(bool(online)), _ptr(out)))
    return out[:w.size]


class Pool(Server):
    """One server per listed device in this process (b2_pool_*); each submit
    goes to the member with the least unfinished work. wait(ticket) returns
    (PdlpResult, info) with info["member"] the index of the server that
    solved it; stats(member) that member's counters."""

    def __init__(self, devices=(0,), hbm_budget_bytes: float = 0.0, round_ms: float = 0.0, max_resident: int = 0,
                 prep_threads: int = 0, grid_nnz: int = 0, grid_slice_ms: float = 0.0, cluster_nnz: int = 0,
                 gpu_scale_nnz: int = 0, **opts):
        so = ServerOpts(float(hbm_budget_bytes), float(round_ms), int(max_resident), int(prep_threads),
                        int(grid_nnz), float(grid_slice_ms), int(cluster_nnz), int(gpu_scale_nnz))
        o = default_opts(**opts)
        dv = np.ascontiguousarray(list(devices), dtype=np.int32)
        h = C.c_void_p()
        _check(lib().b2_pool_create(_ptr(dv), int(dv.size), C.byref(so), C.byref(o), C.byref(h)))
        self._h = h
        self._dims = {}
        self.members = int(dv.size)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().b2_pool_destroy(self._h)
            self._h = C.c_void_p()

    def submit(self, unscaled_form: RangedLP) -> int:
        U = RangedLP.like(unscaled_form)
        t = C.c_int64()
        _check(lib().b2_pool_submit(self._h, C.byref(U.view()), C.byref(t)))
        self._dims[t.value] = (U.m, U.n)
        return t.value

    def submit_file(self, path: str) -> int:
        m, n, _ = lp_file_dims(path)
        t = C.c_int64()
        _check(lib().b2_pool_submit_file(self._h, os.fsencode(path), C.byref(t)))
        self._dims[t.value] = (m, n)
        return t.value

    def wait(self, ticket: int, timeout_s: float = -1.0):
        m, n = self._dims[ticket]
        x = np.zeros(max(n, 1))
        y = np.zeros(max(m, 1))
        r = _Result()
        inf = RequestInfo()
        k = C.c_int32(-1)
        rc = lib().b2_pool_wait(self._h, int(ticket), float(timeout_s), _ptr(x), _ptr(y), C.byref(r), C.byref(inf),
                                C.byref(k))
        if rc == B2_ERR_PENDING:
            return None
        del self._dims[ticket]
        _check(rc)
        info = {k_: getattr(inf, k_) for k_, _ in RequestInfo._fields_}
        info["member"] = k.value
        return _result(r, x[:n], y[:m]), info

    def stats(self, member: int = 0) -> dict:
        st = ServerStats()
        _check(lib().b2_pool_stats_get(self._h, int(member), C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}


# ---------------------------------------------------------- request files
def write_lp(path: str, lp: RangedLP):
    """Stores an LP in the binary request format (A in CSR; b2_lp_write)."""
    lp = RangedLP.like(lp)
    _check(lib().b2_lp_write(os.fsencode(path), C.byref(lp.view())))


def lp_file_dims(path: str):
    m, n, z = C.c_int32(), C.c_int32(), C.c_int64()
    _check(lib().b2_lp_read_dims(os.fsencode(path), C.byref(m), C.byref(n), C.byref(z)))
    return m.value, n.value, z.value


def read_lp(path: str) -> RangedLP:
    """Reads a request file back (A in COO, rows in order)."""
    m, n, z = lp_file_dims(path)
    row = np.zeros(max(z, 1), np.int32); col = np.zeros(max(z, 1), np.int32); val = np.zeros(max(z, 1))
    c = np.zeros(max(n, 1)); l = np.zeros(max(n, 1)); u = np.zeros(max(n, 1))
    rL = np.zeros(max(m, 1)); rU = np.zeros(max(m, 1)); off = C.c_double()
    _check(lib().b2_lp_read(os.fsencode(path), *[_ptr(a) for a in (row, col, val, c, rL, rU, l, u)], C.byref(off)))
    return RangedLP(m, n, row[:z], col[:z], val[:z], c[:n], rL[:m], rU[:m], l[:n], u[:n], off.value)


# ------------------------------------------------------------- host-side prep
def scale(lp: RangedLP, ruiz_passes: int = 10, on_gpu: bool = False):
    """Ruiz + Pock-Chambolle scaling (src/scaling.cpp:25-84). Returns (scaled, Dr, Dc).
    on_gpu: the same computation on the current GPU (b2_scale_gpu), bit for bit."""
    lp = RangedLP.like(lp)
    vs = np.zeros(max(lp.nnz, 1)); cs = np.zeros(max(lp.n, 1)); rls = np.zeros(max(lp.m, 1))
    rus = np.zeros(max(lp.m, 1)); ls = np.zeros(max(lp.n, 1)); us = np.zeros(max(lp.n, 1))
    Dr = np.zeros(max(lp.m, 1)); Dc = np.zeros(max(lp.n, 1))
    v = lp.view()
    fn = lib().b2_scale_gpu if on_gpu else lib().b2_scale
    _check(fn(C.byref(v), ruiz_passes, *[_ptr(a) for a in (vs, cs, rls, rus, ls, us, Dr, Dc)]))
    s = RangedLP(lp.m, lp.n, lp.row, lp.col, vs[:lp.nnz], cs[:lp.n], rls[:lp.m], rus[:lp.m], ls[:lp.n],
                 us[:lp.n], lp.obj_offset)
    return s, Dr[:lp.m], Dc[:lp.n]


def build_pdlp_form(lp: RangedLP):
    """PDLP form of a ranged LP, as build_pdlp_form (src/pdlp.cpp:8-82): equality rows
    first, then one-sided rows as A x >= b (<= rows negated), ranged rows become an
    equality with a bounded slack column, free rows are dropped. Returns
    (form, meta) with meta = (row_perm, row_signs, n_orig, m_orig)."""
    lp = RangedLP.like(lp)
    rL, rU = lp.rL, lp.rU
    eq = [], []
    ineq = [], [], []
    slack = []
    slack_of = {}
    for i in range(lp.m):
        lo, hi = rL[i], rU[i]
        if lo == hi:
            eq[0].append(i); eq[1].append(lo)
        elif np.isfinite(lo) and np.isfinite(hi):
            slack_of[i] = len(slack); slack.append((lo, hi))
            eq[0].append(i); eq[1].append(0.0)
        elif np.isfinite(hi):
            ineq[0].append(i); ineq[1].append(-1.0); ineq[2].append(-hi)
        elif np.isfinite(lo):
            ineq[0].append(i); ineq[1].append(1.0); ineq[2].append(lo)
    row_perm = np.array(eq[0] + ineq[0], np.int64)
    signs = np.array([1.0] * len(eq[0]) + ineq[1])
    pos = np.full(lp.m, -1, np.int64)
    pos[row_perm] = np.arange(row_perm.size)
    p = pos[lp.row]
    keep = p >= 0
    rows = [p[keep]]
    cols = [lp.col[keep]]
    vals = [lp.val[keep] * signs[p[keep]]]
    n2 = lp.n + len(slack)
    for k, i in enumerate(eq[0]):
        if i in slack_of:
            rows.append(np.array([k])); cols.append(np.array([lp.n + slack_of[i]])); vals.append(np.array([-1.0]))
    b = np.array(eq[1] + ineq[2], np.float64)
    rU2 = np.concatenate([np.array(eq[1], np.float64), np.full(len(ineq[0]), np.inf)])
    l2 = np.concatenate([lp.l, np.array([s[0] for s in slack], np.float64)])
    u2 = np.concatenate([lp.u, np.array([s[1] for s in slack], np.float64)])
    c2 = np.concatenate([lp.c, np.zeros(len(slack))])
    form = RangedLP(row_perm.size, n2, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), c2, b,
                    rU2, l2, u2, lp.obj_offset)
    return form, (row_perm, signs, lp.n, lp.m)


def gen_random_lp(m: int, n: int, k: int, seed: int = 0, fp32_values: bool = False) -> RangedLP:
    """Equality-form random LP of the benchmark family (see include/b200_pdlp.h)."""
    z = n * k
    row = np.zeros(z, np.int32); col = np.zeros(z, np.int32); val = np.zeros(z)
    c = np.zeros(n); rL = np.zeros(m); rU = np.zeros(m); l = np.zeros(n); u = np.zeros(n)
    _check(lib().b2_gen_random_lp(m, n, k, seed, int(fp32_values), *[_ptr(a) for a in (row, col, val, c, rL, rU,
                                                                                       l, u)]))
    return RangedLP(m, n, row, col, val, c, rL, rU, l, u)


def batch_family_shapes(count: int, seed: int = 0, m_lo: int = 50, m_hi: int = 5000):
    """Shapes of the uneven batch family: m log-uniform on [m_lo, m_hi],
    n = round(U[2,4] m), nonzeros per column uniform on {4..10}; one derived
    seed per LP. Returns a list of (m, n, k, seed)."""
    rng = np.random.default_rng(seed)
    m = np.exp(rng.uniform(np.log(m_lo), np.log(m_hi), count)).round().astype(int)
    n = np.round(rng.uniform(2.0, 4.0, count) * m).astype(int)
    k = rng.integers(4, 11, count)
    seeds = rng.integers(0, 2**62, count)
    return [(int(a), int(b), int(c), int(d)) for a, b, c, d in zip(m, n, k, seeds)]


def gen_transport(S: int, D: int, seed: int = 0) -> RangedLP:
    """Balanced transportation LP of the benchmark family (see include/b200_pdlp.h)."""
    n, m = S * D, S + D
    row = np.zeros(2 * n, np.int32); col = np.zeros(2 * n, np.int32); val = np.zeros(2 * n)
    c = np.zeros(n); rL = np.zeros(m); rU = np.zeros(m); l = np.zeros(n); u = np.zeros(n)
    _check(lib().b2_gen_transport(S, D, seed, *[_ptr(a) for a in (row, col, val, c, rL, rU, l, u)]))
    return RangedLP(m, n, row, col, val, c, rL, rU, l, u)


def prepare(lp: RangedLP):
    """Host pipeline up to the engine's inputs for an LP without presolve:
    build_pdlp_form -> scale. Returns (unscaled_form, scaled_form, Dr, Dc, meta)."""
    form, meta = build_pdlp_form(lp)
    scaled, Dr, Dc = scale(form)
    return form, scaled, Dr, Dc, meta


def _lp_from_view(v: "_LPView") -> RangedLP:
    """A copy of the arrays a library-owned view points at."""
    def arr(p, n, t):
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(t)), shape=(n,)).copy() if n else np.zeros(0, dtype=t)
    z = int(v.nnz)
    return RangedLP(int(v.m), int(v.n), arr(v.row_idx, z, C.c_int32), arr(v.col_idx, z, C.c_int32),
                    arr(v.val, z, C.c_double), arr(v.c, v.n, C.c_double), arr(v.rL, v.m, C.c_double),
                    arr(v.rU, v.m, C.c_double), arr(v.l, v.n, C.c_double), arr(v.u, v.n, C.c_double),
                    float(v.obj_offset))


class PdlpForm:
    """The PDLP form of a ranged LP built by the library (b2_pdlp_form_build,
    as the reference's build_pdlp_form, src/pdlp.cpp:8-82): .form is the form
    as a RangedLP; extract(x2, y2) maps a point of the form back to the input LP."""

    def __init__(self, lp: RangedLP):
        L = RangedLP.like(lp)
        h = C.c_void_p()
        _check(lib().b2_pdlp_form_build(C.byref(L.view()), C.byref(h)))
        self._h, self.m_in, self.n_in = h, L.m, L.n
        v = _LPView()
        lib().b2_pdlp_form_view(self._h, C.byref(v))
        self.form = _lp_from_view(v)

    def extract(self, x2, y2):
        x = np.zeros(max(self.n_in, 1)); y = np.zeros(max(self.m_in, 1))
        _check(lib().b2_pdlp_form_extract(self._h, _ptr(_vec(x2, self.form.n)), _ptr(_vec(y2, self.form.m)),
                                          _ptr(x), _ptr(y)))
        return x[:self.n_in], y[:self.m_in]

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().b2_pdlp_form_destroy(self._h)
            self._h = C.c_void_p()


class Presolved:
    """b2_presolve: .status (0 reduced, 1 infeasible, 2 unbounded), .reduced
    (a RangedLP); postsolve(x_red, y_red) maps a point of the reduced LP back
    to the original LP, dual values included."""

    def __init__(self, lp: RangedLP):
        L = RangedLP.like(lp)
        h = C.c_void_p()
        st = C.c_int32()
        _check(lib().b2_presolve(C.byref(L.view()), C.byref(h), C.byref(st)))
        self._h, self.status, self.m0, self.n0 = h, int(st.value), L.m, L.n
        v = _LPView()
        lib().b2_presolved_view(self._h, C.byref(v))
        self.reduced = _lp_from_view(v)

    def postsolve(self, x_red, y_red):
        x = np.zeros(max(self.n0, 1)); y = np.zeros(max(self.m0, 1))
        xr = _vec(x_red, self.reduced.n) if self.reduced.n else np.zeros(1)
        yr = _vec(y_red, self.reduced.m) if self.reduced.m else np.zeros(1)
        _check(lib().b2_postsolve(self._h, _ptr(xr), _ptr(yr), _ptr(x), _ptr(y)))
        return x[:self.n0], y[:self.m0]

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().b2_presolved_destroy(self._h)
            self._h = C.c_void_p()


def shape_class(m: int, n: int, nnz: int) -> int:
    """Shape class of an LP (b2_shape_class): size bucket x entries-per-row bucket."""
    return int(lib().b2_shape_class(int(m), int(n), int(nnz)))


def default_tune_table() -> dict:
    """The built-in lane target per shape class (b2_default_tune_table)."""
    t = TuneTable()
    lib().b2_default_tune_table(C.byref(t))
    return {"lane_target": list(t.lane_target), "us_per_attempt": list(t.us_per_attempt)}


def autotune(problems, **opts) -> TuneTable:
    """Runs the shape-class autotuner (b2_batch_autotune) over a list of
    (unscaled, scaled, Dr, Dc) problems on the current GPU; returns the table,
    which Batch / Server accept as tune=..."""
    keep = []
    us, ss, drs, dcs = [], [], [], []
    for (U, S, Dr, Dc) in problems:
        U = RangedLP.like(U)
        S = RangedLP.like(S)
        dr = _vec(Dr, U.m)
        dc = _vec(Dc, U.n)
        keep.extend([U, S, dr, dc])
        us.append(U.view())
        ss.append(S.view())
        drs.append(dr.ctypes.data)
        dcs.append(dc.ctypes.data)
    n = len(us)
    o = default_opts(**opts)
    t = TuneTable()
    _check(lib().b2_batch_autotune(n, (_LPView * n)(*us), (_LPView * n)(*ss), (C.c_void_p * n)(*drs),
                                   (C.c_void_p * n)(*dcs), C.byref(o), C.byref(t)))
    del keep
    return t


def version() -> str:
    return lib().b2_version().decode()
