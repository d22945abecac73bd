"""The allocation-free entry point gs2g_run_rows_noalloc, called through the
C-ABI with ctypes.

It serves callers that must not allocate device memory while they solve
(a framework's memory arena that forbids cudaMalloc/cudaFree in its hot
path, real-time code that cannot take an allocation's implicit
synchronisation): inputs and outputs are the caller's device buffers, and
the sweep kernel's scratch lives in a static device array of the library.
Its results must equal those of the regular entry point (gs2g_run) on the
same rows, on two calls in a row (the second call reuses the static scratch
the first one left behind).

This file is named to be collected last, so a run that stops at the first
failure has run every other test before it.
"""

import ctypes

import numpy as np
import pytest

from conftest import TOL_V_FP64, TOL_V_MIXED

pytestmark = pytest.mark.gpu


class RunOpts(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int), ("tol", ctypes.c_double), ("fixed_iters", ctypes.c_int),
                ("precision", ctypes.c_int), ("start", ctypes.c_int), ("pivot_floor", ctypes.c_double),
                ("n_ctas", ctypes.c_int), ("profile_phases", ctypes.c_int), ("refactor_policy", ctypes.c_int),
                ("refactor_ratio", ctypes.c_double), ("max_reuse", ctypes.c_int), ("rescue", ctypes.c_int),
                ("iters_per_round", ctypes.c_int), ("step_then_check", ctypes.c_int),
                ("step_scaling", ctypes.c_int), ("max_dva", ctypes.c_double), ("max_dvm", ctypes.c_double)]


def _capi():
    from gpusim2grid_b200._native import LIB_PATH
    lib = ctypes.CDLL(str(LIB_PATH))
    f = lib.gs2g_run_rows_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                  ctypes.POINTER(RunOpts), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    lib.gs2g_last_error.restype = ctypes.c_char_p
    return lib


# the 2000-bus grid's per-row workspace (about 1.5 MB in mixed precision,
# 3 MB in FP64) fits the 64 MiB scratch fewer times than the sweep has CTAs,
# so those cases run the clamped CTA count
@pytest.mark.parametrize("grid,n_rows", [("case118_synth", 24), ("case2000_synth", 96)])
@pytest.mark.parametrize("precision,tol_v", [(0, TOL_V_FP64), (1, TOL_V_MIXED)])
def test_noalloc_matches_regular_entry_point(precision, tol_v, grid, n_rows):
    import torch
    from gpusim2grid_b200._native import lib as G
    from gpusim2grid_b200.synthetic import grid_by_name, injection_scenarios

    g = grid_by_name(grid, 0)
    Y, V0, S, _, _, pv, pq = g.as_tuple()
    s = G.Session(0, g.n_bus, Y.indptr.astype(np.int32), Y.indices.astype(np.int32), Y.data, V0, S, pv, pq, 1)
    p, q = injection_scenarios(g, n_rows, seed=9)
    n = p.shape[0]
    # regular entry point: rows from the session's own (allocating) buffers
    s.set_injections(p, q, g.sn_mva)
    s.run(10, 1e-8, False, precision, G.START_VINIT, 0.0, 0, False, 0)
    V_ref, res_ref, st_ref, it_ref = s.results()

    dev = torch.device("cuda", 0)
    v0 = torch.from_numpy(V0.astype(np.complex128)).to(dev)
    sbus = torch.from_numpy(((p + 1j * q) / g.sn_mva).astype(np.complex128)).to(dev)
    capi = _capi()
    opts = RunOpts(max_iter=10, tol=1e-8, fixed_iters=0, precision=precision, start=0, pivot_floor=0.0, n_ctas=0,
                   profile_phases=0, refactor_policy=0, refactor_ratio=0.0, max_reuse=0, rescue=0,
                   iters_per_round=1, step_then_check=0)
    for call in range(2):
        v_out = torch.full((n, g.n_bus), complex("nan+nanj"), dtype=torch.complex128, device=dev)
        res = torch.full((n,), -1.0, dtype=torch.float64, device=dev)
        st = torch.full((n,), -1, dtype=torch.int32, device=dev)
        it = torch.full((n,), -1, dtype=torch.int32, device=dev)
        torch.cuda.synchronize()
        rc = capi.gs2g_run_rows_noalloc(s.handle(), n, v0.data_ptr(), 0, sbus.data_ptr(), g.n_bus,
                                        ctypes.byref(opts), v_out.data_ptr(), res.data_ptr(), st.data_ptr(),
                                        it.data_ptr(), None)
        assert rc == 0, capi.gs2g_last_error()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(st.cpu().numpy(), st_ref)
        np.testing.assert_array_equal(it.cpu().numpy(), it_ref)
        assert np.abs(v_out.cpu().numpy() - V_ref).max() < tol_v, call
        assert np.allclose(res.cpu().numpy(), res_ref, rtol=0, atol=1e-12)
    s.close()


def test_noalloc_rejects_base_chord_and_bad_rounds():
    """Options the allocation-free path cannot honour are refused before any
    launch: the shared-base-factor strategy and an out-of-range round length."""
    import torch
    from gpusim2grid_b200._native import lib as G
    from gpusim2grid_b200.synthetic import grid_by_name

    g = grid_by_name("case118_synth", 0)
    Y, V0, S, _, _, pv, pq = g.as_tuple()
    s = G.Session(0, g.n_bus, Y.indptr.astype(np.int32), Y.indices.astype(np.int32), Y.data, V0, S, pv, pq, 1)
    dev = torch.device("cuda", 0)
    v0 = torch.from_numpy(V0.astype(np.complex128)).to(dev)
    sb = torch.from_numpy(S.astype(np.complex128)).to(dev)
    out = torch.zeros(g.n_bus, dtype=torch.complex128, device=dev)
    res = torch.zeros(1, dtype=torch.float64, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    it = torch.zeros(1, dtype=torch.int32, device=dev)
    capi = _capi()
    for policy, k, word in ((2, 1, b"BASE_CHORD"), (0, 5000, b"iters_per_round")):
        opts = RunOpts(max_iter=10, tol=1e-8, precision=0, refactor_policy=policy, iters_per_round=k)
        rc = capi.gs2g_run_rows_noalloc(s.handle(), 1, v0.data_ptr(), 0, sb.data_ptr(), 0, ctypes.byref(opts),
                                        out.data_ptr(), res.data_ptr(), st.data_ptr(), it.data_ptr(), None)
        assert rc == 1 and word in capi.gs2g_last_error()
    s.close()
