"""The C-ABI shared library loads and exports every symbol include/gs2g.h
declares; GPU-free entry points work through plain ctypes."""

import ctypes
import os
import re

import numpy as np

from gpusim2grid_b200._native import LIB_PATH

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "gs2g.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gs2g_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    lib = ctypes.CDLL(str(LIB_PATH))
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_plan_info_through_ctypes(g118):
    lib = ctypes.CDLL(str(LIB_PATH))

    class Info(ctypes.Structure):
        _fields_ = [("n_bus", ctypes.c_int), ("nnz_y", ctypes.c_int), ("n_pvpq", ctypes.c_int),
                    ("n_pq", ctypes.c_int), ("dim_j", ctypes.c_int), ("nnz_j", ctypes.c_int64),
                    ("nnz_lu", ctypes.c_int64), ("head_dim", ctypes.c_int), ("tail_dim", ctypes.c_int),
                    ("tail_dim_exact", ctypes.c_int), ("n_levels", ctypes.c_int), ("n_supernodes", ctypes.c_int),
                    ("head_madds", ctypes.c_int64), ("schur_madds", ctypes.c_int64),
                    ("dense_madds", ctypes.c_int64), ("plan_ms", ctypes.c_double)]

    Y = g118.Ybus
    ip = np.ascontiguousarray(Y.indptr, dtype=np.int32)
    ix = np.ascontiguousarray(Y.indices, dtype=np.int32)
    pv = np.ascontiguousarray(g118.pv, dtype=np.int32)
    pq = np.ascontiguousarray(g118.pq, dtype=np.int32)
    P = ctypes.POINTER(ctypes.c_int)
    info = Info()
    rc = lib.gs2g_plan_info(g118.n_bus, ip.ctypes.data_as(P), ix.ctypes.data_as(P), pv.ctypes.data_as(P),
                            len(pv), pq.ctypes.data_as(P), len(pq), 1, ctypes.byref(info))
    assert rc == 0
    assert info.dim_j == 117 + 64 and info.head_dim + info.tail_dim == info.dim_j
    # error path: a bad argument returns GS2G_ERR_INVALID with a message
    rc = lib.gs2g_plan_info(0, ip.ctypes.data_as(P), ix.ctypes.data_as(P), pv.ctypes.data_as(P), len(pv),
                            pq.ctypes.data_as(P), len(pq), 1, ctypes.byref(info))
    assert rc == 1
    lib.gs2g_last_error.restype = ctypes.c_char_p
    assert b"plan_info" in lib.gs2g_last_error()
    assert lib.gs2g_version() >= 100
    assert lib.gs2g_max_edits_per_row() == 64


def test_ctypes_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of gs2g_run_opts and gs2g_timings used by the tests
    and shown in INTEGRATION.md have the header's size and field offsets (a
    shorter mirror would let the library read past the caller's struct)."""
    import subprocess
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from test_zz_no_alloc import RunOpts
    src = tmp_path / "layout.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "gs2g.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu\\n", sizeof(gs2g_run_opts), '
                   'offsetof(gs2g_run_opts, iters_per_round), offsetof(gs2g_run_opts, step_then_check), '
                   'sizeof(gs2g_timings)); printf("%zu %zu\\n", offsetof(gs2g_run_opts, step_scaling), '
                   'offsetof(gs2g_run_opts, max_dvm)); return 0; }\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    size, off_k, off_s, _, off_sc, off_vm = map(int, subprocess.run([str(exe)], capture_output=True, text=True,
                                                                    check=True).stdout.split())
    assert ctypes.sizeof(RunOpts) == size
    assert RunOpts.iters_per_round.offset == off_k and RunOpts.step_then_check.offset == off_s
    assert RunOpts.step_scaling.offset == off_sc and RunOpts.max_dvm.offset == off_vm
    doc = open(os.path.join(os.path.dirname(HEADER), "..", "INTEGRATION.md")).read()
    assert '("iters_per_round", I), ("step_then_check", I),' in doc
    assert '("step_scaling", I), ("max_dva", D), ("max_dvm", D)' in doc
