"""Generate tests/golden/reference_golden.npz from the reference's OWN Python
code, to pin the CPU oracle (and through it the engine) to the reference.

    python tests/golden/make_reference_golden.py [path of the reference checkout]

The reference's native library cannot be built here (it needs cuDSS, Eigen and
lightsim2grid), but three pieces of its Python are plain numpy / scipy and run
as they are.  This script loads them from the reference checkout -- it is the
only file of this repository that reads that checkout, and only when run by
hand in a container that has it -- runs them on the seeded synthetic grids
of ``gpusim2grid_b200.synthetic``, and stores inputs and outputs:

* ``tests/python/_jacobian_ref.py: compute_jacobian`` -- the reference test
  suite's MATPOWER Jacobian, at a flat start, at a perturbed voltage and at a
  solution of the 118-bus grid;
* the dense Newton-Raphson of ``tests/python/test_injection_batch.py:
  _lightsim_reference`` (the reference's own CPU check of its injection
  sweep) -- loaded by parsing that file and compiling that one function, since
  the test module itself imports lightsim2grid fixtures -- on the base case at
  several load scales, on N-1 rows (Ybus rebuilt without the branch, not
  through the oracle's trip rule) and on a grid with two half-open branches;
* ``src/gpusim2grid/acpf_nr/_branch_flows.py: compute_branch_flows_cpu`` --
  the branch currents in amperes, open ends included.

The reference's dense NR iterates until ||F||inf < 1e-10 (at most 40 steps),
so its voltages are the converged solutions to that tolerance.
"""

from __future__ import annotations

import ast
import importlib.util
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from gpusim2grid_b200.synthetic import build_ybus, grid_by_name, half_open_variant, n1_branches  # noqa: E402

SCALES = (0.6, 0.8, 1.0, 1.2)
N1_ROWS = 8


def _load_module(path, name):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _load_function(path, fname):
    """Compile one top-level function of a source file, without running the
    rest of the module (its imports need the reference's test fixtures)."""
    with open(path) as fh:
        src = fh.read()
    tree = ast.parse(src, filename=path)
    node = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == fname)
    mod = ast.Module(body=[node], type_ignores=[])
    ns = {"np": np}
    exec(compile(mod, path, "exec"), ns)
    return ns[fname]


def _case(g, Y=None):
    """The dict the reference's dense NR reads (its ieee14_base_case fixture's keys)."""
    Yb, V0, S, _, _, pv, pq = g.as_tuple()
    return dict(n_bus=g.n_bus, Ybus=sp.csr_matrix(Yb if Y is None else Y), pv=np.asarray(pv, dtype=np.int64),
                pq=np.asarray(pq, dtype=np.int64), v_init=V0, Sbus=S)


def main(ref_root):
    jac = _load_module(os.path.join(ref_root, "tests", "python", "_jacobian_ref.py"), "ref_jacobian")
    flows = _load_module(os.path.join(ref_root, "src", "gpusim2grid", "acpf_nr", "_branch_flows.py"),
                         "ref_branch_flows")
    dense_nr = _load_function(os.path.join(ref_root, "tests", "python", "test_injection_batch.py"),
                              "_lightsim_reference")

    g = grid_by_name("case118_synth", 0)
    Y, V0, S, _, _, pv, pq = g.as_tuple()
    pvpq = np.sort(np.concatenate([pv, pq])).astype(np.int64)
    out = dict(pvpq=pvpq, scales=np.asarray(SCALES))

    # the reference's dense NR: base case at several load scales
    V_scaled = dense_nr(None, _case(g), SCALES)
    out["V_scaled"] = V_scaled

    # the reference's Jacobian at a flat start, a perturbed V and a solution
    rng = np.random.default_rng(3)
    Vp = np.abs(V0) * (1 + 0.02 * rng.standard_normal(g.n_bus)) * np.exp(1j * 0.05 * rng.standard_normal(g.n_bus))
    Vsol = V_scaled[SCALES.index(1.0)]
    for name, V in (("flat", V0), ("perturbed", Vp), ("solution", Vsol)):
        J = sp.csr_matrix(jac.compute_jacobian(V, sp.csr_matrix(Y), pvpq, np.asarray(pq, dtype=np.int64)))
        J.sort_indices()
        out[f"V_{name}"] = V
        out[f"J_{name}_data"], out[f"J_{name}_indices"], out[f"J_{name}_indptr"] = J.data, J.indices, J.indptr

    # N-1 rows: Ybus rebuilt from the branch list without the tripped branch
    rows = n1_branches(g)[:N1_ROWS].astype(np.int64)
    V_n1 = np.empty((rows.size, g.n_bus), dtype=np.complex128)
    for r, l in enumerate(rows):
        keep = np.ones(g.n_branch, dtype=bool)
        keep[l] = False
        *_, Yr = build_ybus(g.n_bus, g.branch_from[keep], g.branch_to[keep], g.r[keep], g.x[keep], g.b[keep],
                            g.tap[keep])
        V_n1[r] = dense_nr(None, _case(g, Yr), [1.0])[0]
    out["n1_rows"], out["V_n1"] = rows, V_n1

    # a grid with two half-open branches: its solution and the branch currents
    h = half_open_variant(g, n_open=2, seed=0)
    V_half = dense_nr(None, _case(h), [1.0])[0]
    vn = np.asarray(np.linspace(110.0, 400.0, g.n_bus))
    or_a, ex_a = flows.compute_branch_flows_cpu(V_half, h.branch_from, h.branch_to, h.yff, h.yft, h.ytf, h.ytt,
                                                vn, h.sn_mva)
    out.update(half_open=h.open_branches, V_half=V_half, bus_vn_kv=vn, or_amps=np.asarray(or_a),
               ex_amps=np.asarray(ex_a))
    path = os.path.join(HERE, "reference_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
