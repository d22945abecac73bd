"""The CPU oracle against outputs of the reference's own Python code
(``tests/golden/reference_golden.npz``, written by
``tests/golden/make_reference_golden.py`` from the reference's
``_jacobian_ref.compute_jacobian``, the dense Newton-Raphson of its
``test_injection_batch.py`` and its ``compute_branch_flows_cpu``).  These
pin the oracle's Jacobian, Newton iterates, branch-trip rule and branch
currents to the reference rather than to the oracle itself."""

import os

import numpy as np
import pytest
import scipy.sparse as sp

from gpusim2grid_b200.synthetic import half_open_variant
from oracle import nr_oracle as O

REF = os.path.join(os.path.dirname(__file__), "golden", "reference_golden.npz")


@pytest.fixture(scope="module")
def ref():
    return np.load(REF)


@pytest.mark.parametrize("point", ["flat", "perturbed", "solution"])
def test_jacobian_equals_the_reference_test_suites(g118, ref, point):
    Y, _, _, _, _, pv, pq = g118.as_tuple()
    pvpq, pq_, dim = O.j_layout(g118.n_bus, pv, pq)
    np.testing.assert_array_equal(pvpq, ref["pvpq"])
    Jr = sp.csr_matrix((ref[f"J_{point}_data"], ref[f"J_{point}_indices"], ref[f"J_{point}_indptr"]),
                       shape=(dim, dim))
    J = O.jacobian(Y, ref[f"V_{point}"], pvpq, pq_).tocsr()
    scale = np.abs(Jr.data).max()
    np.testing.assert_allclose(J.toarray(), Jr.toarray(), rtol=0, atol=1e-12 * scale)


def test_newton_solutions_equal_the_references_dense_nr(g118, ref):
    """Same Newton iterates, so the same solutions up to rounding; the
    reference's loop stops at ||F|| < 1e-10, so the oracle is run to that
    tolerance too."""
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    pvpq, pq_, _ = O.j_layout(g118.n_bus, pv, pq)
    for s, Vr in zip(ref["scales"], ref["V_scaled"]):
        assert O.nan_inf_norm(O.mismatch(Y, Vr, S * s, pvpq, pq_)) < 1e-10
        V, st, it, res = O.nr_solve(Y, V0, S * s, pv, pq, 40, 1e-10)
        assert st == O.CONVERGED and res < 1e-10
        assert np.abs(V - Vr).max() < 1e-11, (s, np.abs(V - Vr).max())


def test_branch_trip_rule_equals_the_reference_on_rebuilt_ybus(g118, ref):
    """N-1 rows: the oracle trips the branch on the base Ybus (the
    reference's four-term rule); the reference's dense NR solved a Ybus
    rebuilt without the branch."""
    Y, V0, S, _, _, pv, pq = g118.as_tuple()
    for l, Vr in zip(ref["n1_rows"], ref["V_n1"]):
        Yt = O.trip_branches(Y, [int(l)], g118.branch_from, g118.branch_to, g118.yff, g118.yft, g118.ytf,
                             g118.ytt)
        V, st, _, _ = O.nr_solve(Yt, V0, S, pv, pq, 40, 1e-10)
        assert st == O.CONVERGED
        assert np.abs(V - Vr).max() < 1e-11


def test_half_open_grid_and_branch_currents(g118, ref):
    h = half_open_variant(g118, n_open=2, seed=0)
    np.testing.assert_array_equal(h.open_branches, ref["half_open"])
    Y, V0, S, _, _, pv, pq = h.as_tuple()
    V, st, _, _ = O.nr_solve(Y, V0, S, pv, pq, 40, 1e-10)
    assert st == O.CONVERGED and np.abs(V - ref["V_half"]).max() < 1e-11
    i_or, i_ex = O.branch_currents_amps(ref["V_half"], h.branch_from, h.branch_to, h.yff, h.yft, h.ytf, h.ytt,
                                        ref["bus_vn_kv"], h.sn_mva)
    np.testing.assert_allclose(i_or, ref["or_amps"], rtol=1e-13)
    np.testing.assert_allclose(i_ex, ref["ex_amps"], rtol=1e-13)
    assert np.all(i_ex[h.open_branches] == 0)
    # the power flows the engine reports are these currents times the end voltages
    Sf, St = O.branch_flows(ref["V_half"], h.branch_from, h.branch_to, h.yff, h.yft, h.ytf, h.ytt)
    kv = ref["bus_vn_kv"][h.branch_from]
    np.testing.assert_allclose(np.abs(Sf), i_or * np.abs(ref["V_half"][h.branch_from]) * np.sqrt(3) * kv * 1e-3 /
                               h.sn_mva, rtol=1e-12)
