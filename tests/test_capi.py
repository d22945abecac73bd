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
