"""Build and call the compiled CPU Newton-Raphson (oracle/cpu_nr.cpp).

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__`` (build) and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may use it: it is
the compiled CPU baseline and a fast FP64 checker, never the product path.

``build()`` compiles ``oracle/libcpunr.so`` with g++ (OpenMP, AVX2/FMA
baseline ISA so the library runs on any x86-64-v3 host); ``sweep()`` solves
a batch of rows of one grid and returns (V, status, iters, residual).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_nr.cpp")
LIB = os.path.join(HERE, "libcpunr.so")
CXXFLAGS = ["-O3", "-std=c++17", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared"]

_lib = None


def build(force=False):
    """Compile the library if it is missing or older than its source."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.run(["g++", *CXXFLAGS, SRC, "-o", LIB], check=True)
    return LIB


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = ctypes.CDLL(LIB)
        P, I, D, L = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64
        lib.cpunr_sweep.argtypes = [I, P, P, P, P, P, L, P, I, P, I, I, P, P, P, P, P, P, I, P, P, I, D, I, D,
                                    P, P, P, P, P, ctypes.c_char_p, I]
        lib.cpunr_sweep.restype = I
        lib.cpunr_plan_info.argtypes = [I, P, P, P, I, P, I, D, P]
        lib.cpunr_plan_info.restype = I
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def sweep(Y, V0, Sbus, pv, pq, branches=None, trips=None, sbus_rows=None, max_iter=10, tol=1e-8, threads=0,
          dense_frac=0.4):
    """FP64 flat-start NR (continuous schedule, one step per round) of a
    batch of rows: ``trips`` a list of tripped-branch lists (needs
    ``branches`` = (from, to, yff, yft, ytf, ytt)), ``sbus_rows`` a (rows,
    n_bus) complex array (None: ``Sbus`` for every row).  Returns (V,
    status, iters, residual, plan_ms)."""
    lib = _load()
    import scipy.sparse as sp
    Y = sp.csr_matrix(Y)
    n = Y.shape[0]
    ip = np.ascontiguousarray(Y.indptr, dtype=np.int32)
    ix = np.ascontiguousarray(Y.indices, dtype=np.int32)
    yv = np.ascontiguousarray(Y.data, dtype=np.complex128)
    v0 = np.ascontiguousarray(V0, dtype=np.complex128)
    if sbus_rows is not None:
        sb = np.ascontiguousarray(sbus_rows, dtype=np.complex128)
        n_rows, stride = sb.shape[0], n
    else:
        sb = np.ascontiguousarray(Sbus, dtype=np.complex128)
        n_rows, stride = len(trips), 0
    if trips is not None:
        ptr = np.zeros(len(trips) + 1, dtype=np.int32)
        ptr[1:] = np.cumsum([len(t) for t in trips])
        ids = np.fromiter((int(b) for t in trips for b in t), dtype=np.int32, count=int(ptr[-1]))
        if ids.size == 0:
            ids = np.zeros(1, dtype=np.int32)
        if len(trips) != n_rows:
            raise ValueError("trips and sbus_rows differ in rows")
    else:
        ptr = ids = None
    if branches is not None:
        f, t, yff, yft, ytf, ytt = branches
        f = np.ascontiguousarray(f, dtype=np.int32)
        t = np.ascontiguousarray(t, dtype=np.int32)
        ys = [np.ascontiguousarray(a, dtype=np.complex128) for a in (yff, yft, ytf, ytt)]
        nb = f.size
    else:
        f = t = np.zeros(1, dtype=np.int32)
        ys = [np.zeros(1, dtype=np.complex128)] * 4
        nb = 0
    pv_ = np.ascontiguousarray(pv, dtype=np.int32)
    pq_ = np.ascontiguousarray(pq, dtype=np.int32)
    V = np.empty((n_rows, n), dtype=np.complex128)
    st = np.empty(n_rows, dtype=np.int32)
    it = np.empty(n_rows, dtype=np.int32)
    res = np.empty(n_rows)
    plan_ms = ctypes.c_double(0.0)
    err = ctypes.create_string_buffer(512)
    rc = lib.cpunr_sweep(n, _p(ip), _p(ix), _p(yv), _p(v0), _p(sb), stride, _p(pv_), pv_.size, _p(pq_), pq_.size,
                         nb, _p(f), _p(t), *[_p(a) for a in ys], n_rows,
                         None if ptr is None else _p(ptr), None if ids is None else _p(ids), int(max_iter),
                         float(tol), int(threads), float(dense_frac), _p(V), _p(st), _p(it), _p(res),
                         ctypes.byref(plan_ms), err, len(err))
    if rc != 0:
        raise ValueError(err.value.decode())
    return V, st, it, res, plan_ms.value


def plan_info(Y, pv, pq, dense_frac=0.4):
    """(head pivots, dense tail size, head values, scatter-program length)."""
    import scipy.sparse as sp
    lib = _load()
    Y = sp.csr_matrix(Y)
    out = np.zeros(4, dtype=np.int64)
    rc = lib.cpunr_plan_info(Y.shape[0], _p(np.ascontiguousarray(Y.indptr, dtype=np.int32)),
                             _p(np.ascontiguousarray(Y.indices, dtype=np.int32)),
                             _p(np.ascontiguousarray(pv, dtype=np.int32)), len(pv),
                             _p(np.ascontiguousarray(pq, dtype=np.int32)), len(pq), float(dense_frac), _p(out))
    if rc != 0:
        raise ValueError("plan failed")
    return tuple(int(x) for x in out)
