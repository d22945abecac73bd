"""Generate the golden vectors of tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

The reference's own tests hold no stored results (they compare live against
lightsim2grid, which is not installable here), so these vectors pin the FP64
oracle's outputs on the seeded 118-bus synthetic grid under the reference's
three schedules:
- the flat-start base solve in the single-solve order (step, then test the
  mismatch before the step: ``src/_cpp/acpf_nr.cu:505-561``);
- N-1 rows from a flat start, continuous schedule with one step per round;
- the same rows in rounds of 3 steps (``nb_iter_per_round = 3``);
- the same rows in the chunked schedule (4 fixed steps from the base case);
- rows started from the base case, the first of them tripping nothing (a row
  that starts converged still runs its first round);
- injection rows.
``make_reference_golden.py`` pins the oracle itself to the reference's own
Python code.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gpusim2grid_b200.synthetic import grid_by_name, injection_scenarios, n1_branches  # noqa: E402
from oracle.nr_oracle import contingency_sweep, injection_sweep, nr_solve  # noqa: E402


def main():
    g = grid_by_name("case118_synth", 0)
    Y, V0, S, _, _, pv, pq = g.as_tuple()
    Vb, st, it, res = nr_solve(Y, V0, S, pv, pq, 10, 1e-8, mode="single")
    assert st == 0
    rows = n1_branches(g)[:24]
    bridge = int(np.setdiff1d(np.arange(g.n_branch), n1_branches(g))[0])
    ctg = [[int(b)] for b in rows] + [[bridge], [int(rows[0]), int(rows[1])]]
    f, t = g.branch_from, g.branch_to
    Vc, sc, ic, rc = contingency_sweep(Y, V0, S, pv, pq, ctg, f, t, g.yff, g.yft, g.ytf, g.ytt, 10, 1e-8)
    Vk, sk, ik, rk = contingency_sweep(Y, Vb, S, pv, pq, ctg, f, t, g.yff, g.yft, g.ytf, g.ytt, 4, 1e-8,
                                       mode="fixed")
    V3, s3, i3, r3 = contingency_sweep(Y, V0, S, pv, pq, ctg, f, t, g.yff, g.yft, g.ytf, g.ytt, 10, 1e-8, k=3)
    ctg_b = [[]] + ctg[:8]
    Vbs, sbs, ibs, rbs = contingency_sweep(Y, Vb, S, pv, pq, ctg_b, f, t, g.yff, g.yft, g.ytf, g.ytt, 10, 1e-8)
    p, q = injection_scenarios(g, 8, seed=1)
    Srows = (p + 1j * q) / g.sn_mva
    Vi, si, ii, ri = injection_sweep(Y, V0, Srows, pv, pq, 10, 1e-8)
    np.savez_compressed(os.path.join(HERE, "case118_golden.npz"),
                        V_base=Vb, base_iters=it, ctg_ptr=np.cumsum([0] + [len(c) for c in ctg]),
                        ctg_ids=np.concatenate([np.asarray(c) for c in ctg]).astype(np.int32),
                        V_ctg=Vc, status_ctg=sc, iters_ctg=ic, res_ctg=rc,
                        V_chunked=Vk, status_chunked=sk, res_chunked=rk,
                        V_k3=V3, status_k3=s3, iters_k3=i3,
                        V_base_start=Vbs, status_base_start=sbs, iters_base_start=ibs,
                        p_mw=p, q_mvar=q, V_inj=Vi, status_inj=si, iters_inj=ii)
    print("wrote", os.path.join(HERE, "case118_golden.npz"))


if __name__ == "__main__":
    main()
