"""TEST INFRASTRUCTURE ONLY (the oracle).

ctypes bindings to the two CPU oracles of the PDLP path:

* ``liboracle.so`` -- this repo's plain-C restatement (``pdlp_oracle.c``), serial FP64;
* ``libsovref.so`` -- the reference solver itself, compiled from its own sources
  by ``oracle/Makefile`` together with the flat wrapper ``ref_capi.cpp``.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsovref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libsovref_gpu.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


@dataclass
class LPForm:
    """An LP as the reference's RangedLP holds it (include/ranged_lp.hpp:10-27):
    rL <= A x <= rU, l <= x <= u, min c'x + obj_offset, A in COO."""

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
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.val.size)

    def normalized(self) -> "LPForm":
        return LPForm(int(self.m), int(self.n), _c(self.row, np.int32), _c(self.col, np.int32),
                      _c(self.val, np.float64), _c(self.c, np.float64), _c(self.rL, np.float64),
                      _c(self.rU, np.float64), _c(self.l, np.float64), _c(self.u, np.float64),
                      float(self.obj_offset), dict(self.meta))


# --------------------------------------------------------------- restatement
class _OrLP(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("nnz", C.c_int64),
                ("row", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p),
                ("c", C.c_void_p), ("rL", C.c_void_p), ("rU", C.c_void_p),
                ("l", C.c_void_p), ("u", C.c_void_p), ("obj_offset", C.c_double)]


_rest = None


def restatement():
    global _rest
    if _rest is None:
        if not os.path.exists(RESTATEMENT_SO):
            raise RuntimeError(f"oracle restatement not built: {RESTATEMENT_SO} (run make -C oracle)")
        lib = C.CDLL(RESTATEMENT_SO)
        lib.or_coo_to_csr.argtypes = [C.c_int, C.c_int, C.c_int64, _i32p, _i32p, _f64p, C.c_int, _i32p, _i32p, _f64p]
        lib.or_matvec.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        lib.or_verify.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p,
                                  _f64p, _f64p, C.c_double, _f64p, _f64p, _f64p]
        lib.or_scale.argtypes = [C.c_int, C.c_int, C.c_int64, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                 C.c_int] + [_f64p] * 8
        lib.or_pdlp_run.argtypes = [C.POINTER(_OrLP), C.POINTER(_OrLP), _f64p, _f64p, C.c_int, C.c_int, C.c_double,
                                    _f64p, _f64p, _i32p, _f64p, C.c_void_p, C.c_int]
        lib.or_pdlp_run.restype = C.c_int
        lib.or_gen_random_lp.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, _i32p, _i32p] + [_f64p] * 6
        lib.or_gen_transport.argtypes = [C.c_int, C.c_int, C.c_uint64, _i32p, _i32p] + [_f64p] * 6
        _rest = lib
    return _rest


def gen_random_lp(m: int, n: int, k: int, seed: int, fp32_values: bool = True) -> LPForm:
    """The benchmark's random equality LP (restated generator; the same bits as
    the product's gen_random_lp, pinned by a content digest in the tests)."""
    z = n * k
    row = np.zeros(z, np.int32); col = np.zeros(z, np.int32); val = np.zeros(z)
    c = np.zeros(n); rL = np.zeros(m); rU = np.zeros(m); l = np.zeros(n); u = np.zeros(n)
    if restatement().or_gen_random_lp(m, n, k, seed, int(fp32_values), row, col, val, c, rL, rU, l, u):
        raise ValueError("bad generator sizes")
    return LPForm(m, n, row, col, val, c, rL, rU, l, u, 0.0)


def gen_transport(S: int, D: int, seed: int) -> LPForm:
    """The benchmark's transportation LP, S sources x D sinks (restated generator)."""
    n = S * D
    row = np.zeros(2 * n, np.int32); col = np.zeros(2 * n, np.int32); val = np.zeros(2 * n)
    c = np.zeros(n); rL = np.zeros(S + D); rU = np.zeros(S + D); l = np.zeros(n); u = np.zeros(n)
    if restatement().or_gen_transport(S, D, seed, row, col, val, c, rL, rU, l, u):
        raise ValueError("bad transport sizes")
    return LPForm(S + D, n, row, col, val, c, rL, rU, l, u, 0.0)


def csr(lp: LPForm, transpose: bool = False):
    """CSR(A) or CSR(A^T) with the reference's stable fill order (include/sparse.hpp:24-50)."""
    lp = lp.normalized()
    rows = lp.n if transpose else lp.m
    ptr = np.zeros(rows + 1, np.int32)
    idx = np.zeros(max(lp.nnz, 1), np.int32)
    dat = np.zeros(max(lp.nnz, 1), np.float64)
    restatement().or_coo_to_csr(lp.m, lp.n, lp.nnz, lp.row, lp.col, lp.val, int(transpose), ptr, idx, dat)
    return ptr, idx[:lp.nnz], dat[:lp.nnz]


def matvec(ptr, idx, dat, x):
    rows = ptr.size - 1
    y = np.zeros(max(rows, 1), np.float64)
    restatement().or_matvec(rows, _c(ptr, np.int32), _c(idx, np.int32) if idx.size else np.zeros(1, np.int32),
                            _c(dat, np.float64) if dat.size else np.zeros(1), _c(x, np.float64), y)
    return y[:rows]


def verify(lp: LPForm, x, y):
    """Restated verify() (src/verify.cpp:24-103). Returns dict of the KKT report."""
    lp = lp.normalized()
    ap, ai, av = csr(lp, False)
    tp, ti, tv = csr(lp, True)
    out = np.zeros(7)
    z1 = lambda a, dt: a if a.size else np.zeros(1, dt)  # noqa: E731
    restatement().or_verify(lp.m, lp.n, ap, z1(ai, np.int32), z1(av, np.float64), tp, z1(ti, np.int32),
                            z1(tv, np.float64), lp.c, lp.rL, lp.rU, lp.l, lp.u, lp.obj_offset,
                            _c(x, np.float64), _c(y, np.float64), out)
    return dict(eps_P=out[0], eps_D=out[1], eps_G=out[2], objective=out[3], dual_objective=out[4],
                max_row_violation=out[5], max_bound_violation=out[6])


def scale(lp: LPForm, ruiz_passes: int = 10):
    """Restated scale() (src/scaling.cpp:25-84). Returns (scaled LPForm, Dr, Dc)."""
    lp = lp.normalized()
    vs = np.zeros(max(lp.nnz, 1)); cs = np.zeros(lp.n); rls = np.zeros(lp.m); rus = np.zeros(lp.m)
    ls = np.zeros(lp.n); us = np.zeros(lp.n); Dr = np.zeros(lp.m); Dc = np.zeros(lp.n)
    restatement().or_scale(lp.m, lp.n, lp.nnz, lp.row, lp.col, lp.val if lp.nnz else np.zeros(1), lp.c, lp.rL,
                           lp.rU, lp.l, lp.u, ruiz_passes, vs, cs, rls, rus, ls, us, Dr, Dc)
    s = LPForm(lp.m, lp.n, lp.row, lp.col, vs[:lp.nnz], cs, rls, rus, ls, us, lp.obj_offset)
    return s, Dr, Dc


def _orlp(lp: LPForm):
    keep = [lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u]
    s = _OrLP(lp.m, lp.n, lp.nnz, *[a.ctypes.data for a in keep], lp.obj_offset)
    return s, keep


def pdlp_run(unscaled: LPForm, scaled: LPForm, Dr, Dc, max_iterations=200000, check_every=64, tol=1e-6,
             trace_len: int = 0):
    """Restated pdlp_run + CPU backend (include/pdlp_algo.hpp:49-185, src/pdlp.cpp:97-142)."""
    U, S = unscaled.normalized(), scaled.normalized()
    su, ku = _orlp(U)
    ss, ks = _orlp(S)
    x = np.zeros(max(U.n, 1)); y = np.zeros(max(U.m, 1)); info = np.zeros(4, np.int32); eps = np.zeros(3)
    trace = np.zeros(max(trace_len, 1))
    restatement().or_pdlp_run(C.byref(su), C.byref(ss), _c(Dr, np.float64), _c(Dc, np.float64), max_iterations,
                              check_every, tol, x, y, info, eps, trace.ctypes.data if trace_len else None, trace_len)
    del ku, ks
    res = dict(x=x[:U.n], y=y[:U.m], iterations=int(info[0]), restarts=int(info[1]), converged=bool(info[2]),
               accepted=int(info[3]), eps_P=eps[0], eps_D=eps[1], eps_G=eps[2])
    if trace_len:
        res["trace"] = trace[:min(trace_len, int(info[0]))]
    return res


# ----------------------------------------------------------------- reference
_ref = {}


def reference_available(gpu: bool = False) -> bool:
    return os.path.exists(REF_GPU_SO if gpu else REF_SO)


def reference(gpu: bool = False):
    key = "gpu" if gpu else "cpu"
    if key not in _ref:
        path = REF_GPU_SO if gpu else REF_SO
        if not os.path.exists(path):
            raise RuntimeError(f"reference oracle not built: {path} (run make -C oracle where the reference is)")
        lib = C.CDLL(path)
        vp = C.c_void_p
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_load_mps.restype = vp
        lib.ref_load_mps.argtypes = [C.c_char_p, C.c_int]
        lib.ref_from_arrays.restype = vp
        lib.ref_from_arrays.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                        _f64p, C.c_double, C.c_int]
        lib.ref_free.argtypes = [vp]
        lib.ref_status.argtypes = [vp]
        lib.ref_form_dims.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.ref_form_export.argtypes = [vp, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                        C.POINTER(C.c_double)]
        lib.ref_scaling_export.argtypes = [vp, _f64p, _f64p]
        lib.ref_scale_arrays.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p,
                                         _f64p] + [_f64p] * 8
        for fn in (lib.ref_solve_pdhg, lib.ref_solve_pdhg_gpu):
            fn.argtypes = [vp, C.c_int, C.c_int, C.c_double, _f64p, _f64p, _i32p, _f64p, C.POINTER(C.c_double)]
        lib.ref_verify_form.argtypes = [vp, C.c_int, _f64p, _f64p, _f64p]
        lib.ref_finish.argtypes = [vp, _f64p, _f64p, _f64p]
        lib.ref_solve_mps.argtypes = [C.c_char_p, C.c_double, C.c_int, _f64p, C.c_char_p, C.c_int]
        lib.ref_solve_simplex_mps.argtypes = [C.c_char_p, C.c_double, _f64p, C.c_char_p, C.c_int]
        lib.ref_write_mps.argtypes = [vp, C.c_char_p]
        _ref[key] = lib
    return _ref[key]


class RefProblem:
    """One LP pushed through the reference pipeline up to the PDLP stage:
    to_ranged_lp -> presolve -> build_pdlp_form -> scale (src/solve.cpp:150-195)."""

    ORIGINAL, PDLP_FORM, SCALED, PRESOLVED = 0, 1, 2, 3

    def __init__(self, handle, lib):
        if not handle:
            raise RuntimeError("reference: " + lib.ref_last_error().decode())
        self.h = handle
        self.lib = lib

    @classmethod
    def from_mps(cls, path: str, use_presolve: bool = True, gpu: bool = False):
        lib = reference(gpu)
        return cls(lib.ref_load_mps(path.encode(), int(use_presolve)), lib)

    @classmethod
    def from_form(cls, lp: LPForm, use_presolve: bool = True, gpu: bool = False):
        lib = reference(gpu)
        lp = lp.normalized()
        z = lambda a, dt: a if a.size else np.zeros(1, dt)  # noqa: E731
        return cls(lib.ref_from_arrays(lp.m, lp.n, lp.nnz, z(lp.row, np.int32), z(lp.col, np.int32),
                                       z(lp.val, np.float64), lp.c, lp.rL, lp.rU, lp.l, lp.u, lp.obj_offset,
                                       int(use_presolve)), lib)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_free(self.h)
            self.h = None

    @property
    def status(self) -> int:
        return self.lib.ref_status(self.h)

    def form(self, which: int) -> LPForm:
        m, n, z = C.c_int(), C.c_int(), C.c_int()
        self.lib.ref_form_dims(self.h, which, C.byref(m), C.byref(n), C.byref(z))
        m, n, z = m.value, n.value, z.value
        row = np.zeros(max(z, 1), np.int32); col = np.zeros(max(z, 1), np.int32); val = np.zeros(max(z, 1))
        c = np.zeros(max(n, 1)); rL = np.zeros(max(m, 1)); rU = np.zeros(max(m, 1))
        l = np.zeros(max(n, 1)); u = np.zeros(max(n, 1)); off = C.c_double()
        self.lib.ref_form_export(self.h, which, row, col, val, c, rL, rU, l, u, C.byref(off))
        return LPForm(m, n, row[:z], col[:z], val[:z], c[:n], rL[:m], rU[:m], l[:n], u[:n], off.value)

    def scaling(self):
        f = self.form(self.PDLP_FORM)
        Dr = np.zeros(max(f.m, 1)); Dc = np.zeros(max(f.n, 1))
        self.lib.ref_scaling_export(self.h, Dr, Dc)
        return Dr[:f.m], Dc[:f.n]

    def solve_pdhg(self, max_iterations=200000, check_every=64, tol=1e-6, gpu=False):
        f = self.form(self.PDLP_FORM)
        x = np.zeros(max(f.n, 1)); y = np.zeros(max(f.m, 1)); info = np.zeros(3, np.int32); eps = np.zeros(3)
        sec = C.c_double()
        fn = self.lib.ref_solve_pdhg_gpu if gpu else self.lib.ref_solve_pdhg
        rc = fn(self.h, max_iterations, check_every, tol, x, y, info, eps, C.byref(sec))
        if rc:
            raise RuntimeError("reference solve_pdhg: " + self.lib.ref_last_error().decode())
        return dict(x=x[:f.n], y=y[:f.m], iterations=int(info[0]), restarts=int(info[1]), converged=bool(info[2]),
                    eps_P=eps[0], eps_D=eps[1], eps_G=eps[2], seconds=sec.value)

    def verify_form(self, which, x, y):
        out = np.zeros(5)
        self.lib.ref_verify_form(self.h, which, _c(x, np.float64), _c(y, np.float64), out)
        return dict(eps_P=out[0], eps_D=out[1], eps_G=out[2], objective=out[3], dual_objective=out[4])

    def finish(self, x2, y2):
        out = np.zeros(4)
        if self.lib.ref_finish(self.h, _c(x2, np.float64), _c(y2, np.float64), out):
            raise RuntimeError("reference finish: " + self.lib.ref_last_error().decode())
        return dict(objective=out[0], eps_P=out[1], eps_D=out[2], eps_G=out[3])

    def write_mps(self, path: str):
        if self.lib.ref_write_mps(self.h, path.encode()):
            raise RuntimeError("reference write_mps failed")


def ref_scale(lp: LPForm):
    """The reference's own scale() on an array form (src/scaling.cpp:25-84)."""
    lib = reference()
    lp = lp.normalized()
    vs = np.zeros(max(lp.nnz, 1)); cs = np.zeros(lp.n); rls = np.zeros(lp.m); rus = np.zeros(lp.m)
    ls = np.zeros(lp.n); us = np.zeros(lp.n); Dr = np.zeros(lp.m); Dc = np.zeros(lp.n)
    lib.ref_scale_arrays(lp.m, lp.n, lp.nnz, lp.row, lp.col, lp.val, lp.c, lp.rL, lp.rU, lp.l, lp.u,
                         vs, cs, rls, rus, ls, us, Dr, Dc)
    return LPForm(lp.m, lp.n, lp.row, lp.col, vs[:lp.nnz], cs, rls, rus, ls, us, lp.obj_offset), Dr, Dc


def ref_solve_simplex_mps(path: str, time_limit: float = 600.0):
    lib = reference()
    out = np.zeros(6)
    buf = C.create_string_buffer(256)
    if lib.ref_solve_simplex_mps(path.encode(), time_limit, out, buf, 256):
        raise RuntimeError("reference simplex: " + lib.ref_last_error().decode())
    return dict(objective=out[0], eps_P=out[1], eps_D=out[2], eps_G=out[3], iterations=int(out[4]),
                seconds=out[5], status=buf.value.decode())


def ref_solve_mps(path: str, tol=1e-6, max_iterations=500000, gpu=False):
    lib = reference(gpu)
    out = np.zeros(6)
    buf = C.create_string_buffer(256)
    if lib.ref_solve_mps(path.encode(), tol, max_iterations, out, buf, 256):
        raise RuntimeError("reference solve_mps: " + lib.ref_last_error().decode())
    st, _, eng = buf.value.decode().partition("|")
    return dict(objective=out[0], eps_P=out[1], eps_D=out[2], eps_G=out[3], iterations=int(out[4]),
                seconds=out[5], status=st, engine=eng)
