"""The compiled CPU Newton-Raphson (oracle/cpu_nr.cpp, the bench's CPU
baseline and a fast FP64 checker) against the numpy oracle: the same
statuses, iteration counts and voltages (to rounding) on N-1 rows with
islanding outages, injection rows, a NaN row, and half-open branches."""

import numpy as np
import pytest

from gpusim2grid_b200.synthetic import half_open_variant, injection_scenarios, n1_branches
from oracle import cpu_nr
from oracle import nr_oracle as O


def _br(g):
    return (g.branch_from, g.branch_to, g.yff, g.yft, g.ytf, g.ytt)


def test_n1_rows_with_islanding_equal_the_oracle(g118):
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    rows = [[b] for b in range(g118.n_branch)] + [[0, 1], [3, 3], []]
    V, st, it, res, _ = cpu_nr.sweep(Y, V0, S, pv, pq, branches=_br(g118), trips=rows, threads=2)
    Vo, so, io, ro = O.contingency_sweep(Y, V0, S, pv, pq, rows, *_br(g118), 10, 1e-8)
    np.testing.assert_array_equal(st, so)
    np.testing.assert_array_equal(it, io)
    ok = so != O.NOT_SIMULATED
    assert (~ok).sum() > 0 and np.all(np.isnan(V[~ok]))
    assert np.abs(V[ok] - Vo[ok]).max() < 1e-12
    np.testing.assert_allclose(res[ok], ro[ok], rtol=0, atol=1e-12)


def test_injection_rows_and_a_nan_row(g118):
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    p, q = injection_scenarios(g118, 12, seed=4)
    sb = (p + 1j * q) / g118.sn_mva
    sb[5, pq[3]] = np.nan
    V, st, it, _, _ = cpu_nr.sweep(Y, V0, S, pv, pq, sbus_rows=sb, threads=3)
    Vo, so, io, _ = O.injection_sweep(Y, V0, sb, pv, pq, 10, 1e-8)
    np.testing.assert_array_equal(st, so)
    np.testing.assert_array_equal(it, io)
    assert st[5] == O.DIVERGED
    ok = so == O.CONVERGED
    assert np.abs(V[ok] - Vo[ok]).max() < 1e-12


def test_half_open_branches_equal_the_oracle(g118):
    h = half_open_variant(g118, n_open=2, seed=0)
    Y, V0, S, _, _, pv, pq = h.as_tuple()
    lo = [int(x) for x in h.open_branches]
    rows = [[lo[0]], lo, [lo[1], int(n1_branches(h)[0])]]
    V, st, it, _, _ = cpu_nr.sweep(Y, V0, S, pv, pq, branches=_br(h), trips=rows, threads=1)
    Vo, so, io, _ = O.contingency_sweep(Y, V0, S, pv, pq, rows, *_br(h), 10, 1e-8)
    np.testing.assert_array_equal(st, so)
    np.testing.assert_array_equal(it, io)
    assert np.abs(V - Vo).max() < 1e-12


def test_2000_bus_rows_equal_the_oracle(g2000):
    Y, V0, S, _, _, pv, pq = g2000.as_tuple()
    rows = [[int(b)] for b in n1_branches(g2000)[::400]]
    V, st, it, _, _ = cpu_nr.sweep(Y, V0, S, pv, pq, branches=_br(g2000), trips=rows)
    Vo, so, io, _ = O.contingency_sweep(Y, V0, S, pv, pq, rows, *_br(g2000), 10, 1e-8)
    np.testing.assert_array_equal(st, so)
    np.testing.assert_array_equal(it, io)
    assert np.abs(V - Vo).max() < 1e-11


def test_bad_branch_id_is_refused(g118):
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    with pytest.raises(ValueError, match="out of range"):
        cpu_nr.sweep(Y, V0, S, pv, pq, branches=_br(g118), trips=[[g118.n_branch]])
