"""The C-ABI library without a GPU: it loads, exports what include/b200_pdlp.h
declares, and rejects malformed input with the documented status codes."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import b200pdlp as B
from conftest import ROOT, gpu_available, load_fixture


def declared_functions():
    src = open(os.path.join(ROOT, "include", "b200_pdlp.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(b2_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = B.lib()
    names = declared_functions()
    assert len(names) >= 12
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(B.EXPORTED)


def test_version_and_defaults():
    assert "sm_100a" in B.version()
    o = B.default_opts()
    assert (o.max_iterations, o.check_every, o.tol) == (200000, 64, 1e-6)
    assert o.precision == B.PREC_MIXED


def _view_args(U, S):
    return B.RangedLP.like(U), B.RangedLP.like(S)


def test_rejects_out_of_range_index():
    U, S, Dr, Dc = load_fixture("afiro")
    U2 = B.RangedLP.like(U)
    U2.col = U2.col.copy()
    U2.col[0] = U.n + 5
    with pytest.raises(B.B2Error) as e:
        B.solve_pdhg_gpu(U2, S, Dr, Dc)
    assert e.value.code == B.B2_ERR_INVALID


def test_rejects_nonfinite_value():
    U, S, Dr, Dc = load_fixture("afiro")
    U2 = B.RangedLP.like(U)
    U2.val = U2.val.copy()
    U2.val[1] = np.nan
    with pytest.raises(B.B2Error) as e:
        B.solve_pdhg_gpu(U2, S, Dr, Dc)
    assert e.value.code == B.B2_ERR_NONFINITE
    U3 = B.RangedLP.like(U)
    U3.c = U3.c.copy()
    U3.c[0] = np.inf
    with pytest.raises(B.B2Error) as e:
        B.solve_pdhg_gpu(U3, S, Dr, Dc)
    assert e.value.code == B.B2_ERR_NONFINITE


def test_rejects_non_pdlp_form():
    """A <= row (rL = -inf) is not a PDLP-form row (src/pdlp.cpp:59-62)."""
    U, S, Dr, Dc = load_fixture("afiro")
    U2 = B.RangedLP.like(U)
    U2.rL = U2.rL.copy()
    U2.rL[0] = -np.inf
    with pytest.raises(B.B2Error) as e:
        B.solve_pdhg_gpu(U2, S, Dr, Dc)
    assert e.value.code == B.B2_ERR_NONFINITE


def test_rejects_inconsistent_scaling():
    U, S, Dr, Dc = load_fixture("afiro")
    S2 = B.RangedLP.like(S)
    S2.c = S2.c * 2.0 + 1.0
    with pytest.raises(B.B2Error) as e:
        B.solve_pdhg_gpu(U, S2, Dr, Dc)
    assert e.value.code == B.B2_ERR_INVALID


@pytest.mark.skipif(gpu_available(), reason="this box has a GPU")
def test_no_device_is_reported_not_hidden():
    """No CPU fallback: without a device the solve fails loudly."""
    U, S, Dr, Dc = load_fixture("afiro")
    with pytest.raises(B.B2Error) as e:
        B.solve_pdhg_gpu(U, S, Dr, Dc)
    assert e.value.code in (B.B2_ERR_NO_DEVICE, B.B2_ERR_CUDA)


def test_stop_flag_word_layout():
    f = B.StopFlag()
    assert not f.is_set()
    f.set()
    assert C.c_int32.from_address(f.ptr).value == 1


def test_noalloc_rejects_lp_above_its_static_limit():
    """The allocation-free entry point refuses, before any GPU work, an LP whose
    device working set exceeds its 32 MiB static array."""
    lp = B.gen_random_lp(60000, 180000, 6, 1, True)
    U, S, Dr, Dc, _ = B.prepare(lp)
    o = B.default_opts()
    r = B._Result()
    uv, sv = U.view(), S.view()
    rc = B.lib().b2_solve_pdhg_gpu_noalloc(C.byref(uv), C.byref(sv), Dr.ctypes.data, Dc.ctypes.data, C.byref(o),
                                            None, None, C.byref(r))
    assert rc == B.B2_ERR_UNSUPPORTED
    assert "32 MiB" in B.lib().b2_last_error().decode()


C_CLIENT = r"""
#include <stdio.h>
#include <string.h>
#include "b200_pdlp.h"

int main(void) {
    /* a plain C caller: version, options, the shard plan and a host-only layout digest */
    b2_solve_opts o;
    b2_default_opts(&o);
    if (o.check_every != 64) return 10;
    int64_t work[5] = {5, 9, 1, 9, 3};
    int32_t rank_of[5];
    if (b2_shard_plan(work, 5, 2, 0, rank_of) != B2_OK) return 11;
    /* longest first: 9 -> 0, 9 -> 1, 5 -> 0, 3 -> 1, 1 -> 1 */
    const int32_t want[5] = {0, 0, 1, 1, 1};
    if (memcmp(rank_of, want, sizeof(want)) != 0) return 12;
    if (b2_request_work(3, 4, 10) != 27) return 13;
    /* min x0 + x1 s.t. x0 + x1 = 1, 0 <= x <= 1 (PDLP form, no scaling) */
    int32_t row[2] = {0, 0}, col[2] = {0, 1};
    double val[2] = {1.0, 1.0}, c[2] = {1.0, 1.0}, rl[1] = {1.0}, ru[1] = {1.0}, l[2] = {0.0, 0.0},
           u[2] = {1.0, 1.0}, dr[1] = {1.0}, dc[2] = {1.0, 1.0};
    b2_lp_view U = {1, 2, 2, row, col, val, c, rl, ru, l, u, 0.0};
    uint64_t d1 = 0, d2 = 0;
    if (b2_layout_digest(&U, &U, dr, dc, 1, 1, &d1) != B2_OK) return 14;
    if (b2_layout_digest(&U, &U, dr, dc, 4, 1, &d2) != B2_OK || d1 != d2) return 15;
    col[1] = 7; /* out of range: rejected on the host, with a message */
    if (b2_layout_digest(&U, &U, dr, dc, 1, 1, &d1) != B2_ERR_INVALID) return 16;
    if (strstr(b2_last_error(), "entry 1") == NULL) return 17;
    printf("c client ok: %s\n", b2_version());
    return 0;
}
"""


def test_header_compiles_as_c_and_a_c_client_runs(tmp_path):
    """include/b200_pdlp.h is a C header (C99, no C++), and the library is
    usable from C: host-only calls run here without a GPU."""
    import subprocess
    src = tmp_path / "client.c"
    src.write_text(C_CLIENT)
    exe = tmp_path / "client"
    libdir = os.path.dirname(B.LIB_PATH)
    cmd = ["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"), str(src),
           "-o", str(exe), "-L", libdir, "-lb200pdlp", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "c client ok" in r.stdout
