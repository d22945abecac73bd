"""The chord sweep (several rows per CTA in lockstep on the shared base
factor, hand-off of the rows that need their own LU to the single-row
sweep) with plain chord steps must take the single-row sweep's decisions:
the same statuses, Newton steps and factorizations per row, and the same
voltages within the mixed-precision bar.  Covers the hand-off, islanded
rows, branch loading at eviction and fewer rows than slots.  With Broyden
steps (the default) the rows converge to the same solutions as plain FP64
Newton, with the same statuses, in no more Newton steps than the chord."""

import numpy as np
import pytest

from conftest import TOL_V_MIXED
from gpusim2grid_b200 import ContingencyAnalysisGPU, InjectionSweepGPU, RowStatus, ScenarioSweepGPU
from gpusim2grid_b200.synthetic import injection_scenarios, n1_branches, scenario_outages

pytestmark = pytest.mark.gpu


CHORD, SINGLE, BROYDEN = 1, 0, 2


def _both(f):
    """(plain chord, single-row) results of the facade's current rows."""
    out = []
    for mode in (CHORD, SINGLE):
        f.session.set_chord(mode)
        f.compute()
        out.append((f.V_results, f.get_row_status(), f.get_row_iterations(), f.get_row_factorizations()))
    f.session.set_chord(BROYDEN)
    return out


def _same(chord, single, tol):
    (Vc, sc, ic, fc), (Vs, ss, is_, fs) = chord, single
    np.testing.assert_array_equal(sc, ss)
    np.testing.assert_array_equal(ic, is_)
    np.testing.assert_array_equal(fc, fs)
    ok = sc == RowStatus.CONVERGED
    if ok.any():
        assert np.abs(Vc[ok] - Vs[ok]).max() < tol
    assert np.all(np.isnan(Vc[sc == RowStatus.NOT_SIMULATED]))


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_chord_n1_matches_single_row(g118, precision):
    ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=10,
                                scheduling="continuous", tol=1e-8, start="base", strategy="base_chord")
    ca.set_branch_data(*g118.branch_data())
    ca.add_contingencies_by_branch_id([[b] for b in range(g118.n_branch)])  # bridges island: not simulated
    chord, single = _both(ca)
    _same(chord, single, TOL_V_MIXED if precision == "mixed" else 1e-9)
    assert (chord[1] == RowStatus.NOT_SIMULATED).any()
    assert (chord[3] > 0).any() and (chord[3] == 0).any()  # some rows were handed off, some stayed


def test_chord_injections_and_outages_with_flows(g118):
    rng = np.random.default_rng(2)
    sw = ScenarioSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=10,
                          scheduling="continuous", tol=1e-8, start="base", strategy="base_chord")
    sw.set_branch_data(*g118.branch_data())
    p, q = injection_scenarios(g118, 301, seed=9)  # not a multiple of the slots per CTA
    sw.set_injections(p, q, g118.sn_mva)
    sw.set_topology(scenario_outages(g118, 301, max_trips=2, seed=10))
    sw.set_branch_limits(rng.uniform(50.0, 300.0, g118.n_branch), g118.sn_mva)
    out = []
    for mode in (CHORD, SINGLE):
        sw.session.set_chord(mode)
        sw.compute()
        out.append((sw.V_results, sw.get_row_status(), sw.get_row_iterations(), sw.get_row_factorizations(),
                    sw.branch_loading()))
    _same(out[0][:4], out[1][:4], TOL_V_MIXED)
    (lc, nc, mc), (ls, ns, ms) = out[0][4], out[1][4]
    ok = out[0][1] == RowStatus.CONVERGED
    np.testing.assert_allclose(lc[ok], ls[ok], rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(nc, ns)
    assert np.all(np.isnan(lc[~ok]))


def test_chord_fewer_rows_than_slots(g118):
    p, q = injection_scenarios(g118, 3, seed=1)
    sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=10,
                           scheduling="continuous", tol=1e-8, start="base", strategy="base_chord")
    sw.set_injections(p, q, g118.sn_mva)
    chord, single = _both(sw)
    _same(chord, single, TOL_V_MIXED)
    assert np.all(chord[1] == RowStatus.CONVERGED)


def test_chord_given_starts_selection_and_rescue(g118):
    """Per-row starts through the chord sweep, as in the single-row sweep:
    NaN starts begin from the base case (start selection) and, having begun
    from the rescue voltage, are not restarted; near-solution starts (the
    solutions perturbed) keep their own start, and with a one-step budget
    they end unconverged there and are rescued from the base case."""
    p, q = injection_scenarios(g118, 64, seed=12)
    ref = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="fp64", nb_iter=10,
                            scheduling="continuous", tol=1e-8, start="base", strategy="refactor_every")
    ref.set_injections(p, q, g118.sn_mva)
    ref.compute()
    sw = InjectionSweepGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="mixed", nb_iter=1,
                           scheduling="continuous", tol=1e-8, start="base", strategy="base_chord")
    sw.set_injections(p, q, g118.sn_mva)
    sw.fallback = None  # the sweep's own statuses and counters, no FP64 re-solve after it
    rng = np.random.default_rng(5)
    V0 = ref.V_results * np.exp(1j * rng.uniform(-1e-5, 1e-5, ref.V_results.shape))
    V0[::3] = np.nan
    sw.set_start_voltages(V0)
    out, counts = [], []
    for mode in (CHORD, SINGLE):
        sw.session.set_chord(mode)
        sw.compute()
        out.append((sw.V_results, sw.get_row_status(), sw.get_row_iterations(), sw.get_row_factorizations()))
        t = sw.session.timings()
        counts.append((t["n_base_start"], t["n_rescued"]))
    _same(out[0], out[1], TOL_V_MIXED)
    n_nan = len(range(0, 64, 3))
    assert counts[0] == counts[1]
    assert counts[0][0] == n_nan                 # only the NaN rows began from the base case
    assert 0 < counts[0][1] <= 64 - n_nan       # rescued rows are among those that kept their start


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_broyden_steps_reach_the_fp64_solutions(g118, precision):
    """Broyden steps on the base factor: N-1 rows and injection + outage rows
    converge to plain FP64 Newton's solutions with the same statuses, in
    fewer Newton steps than the plain chord."""
    ref = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, precision="fp64", nb_iter=10,
                                 scheduling="continuous", tol=1e-8, start="flat", strategy="refactor_every")
    ca = ContingencyAnalysisGPU(g118.as_tuple(), init_from_n_powerflow=False, precision=precision, nb_iter=10,
                                scheduling="continuous", tol=1e-8, start="base", strategy="base_chord")
    rows = [[b] for b in range(g118.n_branch)]
    for f in (ref, ca):
        f.set_branch_data(*g118.branch_data())
        f.add_contingencies_by_branch_id(rows)
    ref.compute()
    its = {}
    for mode in (CHORD, BROYDEN):
        ca.session.set_chord(mode)
        ca.compute()
        np.testing.assert_array_equal(ca.get_row_status(), ref.get_row_status())
        ok = ref.get_row_status() == RowStatus.CONVERGED
        # another iteration stopped at the same ||F|| tolerance: the |dV| bar of the metric
        assert np.abs(ca.V_results[ok] - ref.V_results[ok]).max() < TOL_V_MIXED
        its[mode] = ca.get_row_iterations()[ok].sum()
    assert its[BROYDEN] < its[CHORD]
