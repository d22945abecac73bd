"""Single AC power flow on the GPU: ``acpf_nr_gpu`` and ``AcPfGPU``.

Array-tuple mode of the reference's ``AcPfGPU`` (``src/gpusim2grid/acpf_nr/gpu_facade.py:31-331``)
and its ``acpf_nr_gpu`` binding (``src/_cpp/python_bindings.cpp:1266-1285``).  The
bare ``[pvpq | pq]`` system is solved; ``slack_ids`` / ``slack_weights`` are
accepted and ignored there, as in the reference (``src/_cpp/acpf_nr.cu:1732-1733``).

A single solve runs as a one-row batch on the same persistent kernel as the
sweeps (one CTA), so its result is also exported zero-copy by ``v_dlpack()``.
"""

from __future__ import annotations

import time

import numpy as np

from ._common import (AcPfTimings, grid_arrays, make_session, normalize_device, resolve_precision, RowStatus)
from ._native import lib

__all__ = ["AcPfGPU", "acpf_nr_gpu"]


class AcPfGPU:
    """Single-system AC Newton–Raphson on the GPU.

    Parameters
    ----------
    grid : tuple
        ``(Ybus, Vinit, Sbus, slack_ids, slack_weights, pv, pq)``.
    precision : {"fp64", "mixed"}
    max_iter, tol : int, float
    device : None | int | "cuda" | "cuda:N"
    init_from_n_powerflow : bool, default True
        Trust ``Vinit`` as already solved: validate ``||F(Vinit)||inf < tol``
        once (``RuntimeError`` otherwise) and skip the Newton loop.  With False
        the GPU iterates from ``Vinit``.
    scaling_max_voltage_change, max_dVa, max_dVm
        The reference's MaxVoltageChange step scaling: True multiplies every
        Newton step by alpha <= 1 so that max|dtheta| <= max_dVa and
        max|dVm| <= max_dVm (defaults 0.5 rad / 0.1 pu).  None / False: off.
    """

    def __init__(self, grid, *, precision="fp64", max_iter=10, tol=1e-8, device=None,
                 init_from_n_powerflow=True, scaling_max_voltage_change=None, max_dVa=None, max_dVm=None,
                 **_ignored):
        d = grid_arrays(grid)
        self._d = d
        self._prec = resolve_precision(precision)
        self.max_iter = int(max_iter)
        self.tol = float(tol)
        # MaxVoltageChange step scaling (src/gpusim2grid/acpf_nr/gpu_facade.py:100-121):
        # None (no grid configuration to inherit in array-tuple mode) is off
        self._scaling = dict(step_scaling=bool(scaling_max_voltage_change),
                             max_dva=0.0 if max_dVa is None else float(max_dVa),
                             max_dvm=0.0 if max_dVm is None else float(max_dVm))
        self._s = make_session(d, device)
        self._vm_fixed = None
        self._sbus = d["Sbus"].copy()
        self._push_sbus(self._sbus)
        if init_from_n_powerflow:
            t = self._run(d["Vinit"], max_iter=0, fixed=True)
            if not (t.residual < self.tol):
                raise RuntimeError(f"init_from_n_powerflow: ||F(Vinit)||inf = {t.residual:.3e} is not below "
                                   f"tol = {self.tol:.1e}; pass init_from_n_powerflow=False to solve from Vinit")
            t.converged = True
            self._timings = t
        else:
            self._timings = self._run(d["Vinit"], self.max_iter, False)

    def _push_sbus(self, sbus):
        s = np.asarray(sbus, dtype=np.complex128).reshape(1, -1)
        self._s.set_injections(s.real.copy(), s.imag.copy(), 1.0)

    def _run(self, V0, max_iter, fixed, tol=None):
        t0 = time.perf_counter()
        self._s.set_start_rows(np.asarray(V0, dtype=np.complex128).reshape(1, -1))
        # a free-running solve takes the reference's single-solve order: each
        # step is taken, then the mismatch before it decides convergence
        self._s.run(int(max_iter), float(self.tol if tol is None else tol), bool(fixed), self._prec,
                    lib.START_ROWS, step_then_check=not fixed, **self._scaling)
        tm = self._s.timings()
        _, res, st, it = self._s.results()
        return AcPfTimings(converged=int(st[0]) == RowStatus.CONVERGED, nb_iter=int(it[0]),
                           residual=float(res[0]), t_plan_ms=tm["plan_ms"], t_kernel_ms=tm["kernel_ms"],
                           t_total_ms=(time.perf_counter() - t0) * 1e3)

    def solve(self):
        """The solved complex voltage vector (host copy)."""
        return self._s.results()[0][0].copy()

    def resolve(self, Vinit, Sbus=None, *, max_iter=None, tol=None):
        """Solve again from ``Vinit`` reusing the symbolic analysis; ``Sbus``
        None keeps the current injections.  Returns this solve's timings."""
        self._vm_setpoints()
        if Sbus is not None:
            self._sbus = np.ascontiguousarray(Sbus, dtype=np.complex128).reshape(-1)
            self._push_sbus(self._sbus)
        mi = self.max_iter if max_iter is None else int(max_iter)
        self._timings = self._run(Vinit, mi, False, tol)
        return self._timings

    def ac_pf(self, Vinit, max_iter, tol):
        """lightsim2grid's ``ac_pf(Vinit, max_iter, tol)`` call shape: writes
        the voltage set-points into |V| at PV/slack buses, solves, and returns
        the voltage or an empty array when it did not converge."""
        mask, vm = self._vm_setpoints()
        V = np.array(Vinit, dtype=np.complex128)
        V[mask] = vm[mask] * np.exp(1j * np.angle(V[mask]))
        t = self.resolve(V, max_iter=max_iter, tol=tol)
        return self.solve() if t.converged else np.zeros(0, dtype=np.complex128)

    def _vm_setpoints(self):
        if self._vm_fixed is None:
            mask = np.ones(self._d["n_bus"], dtype=bool)
            mask[self._d["pq"]] = False
            self._vm_fixed = (mask, np.abs(self.solve()))
        return self._vm_fixed

    def v_dlpack(self):
        """Zero-copy DLPack capsule of the solved voltage, shape (1, n_bus)."""
        return self._s.dlpack("v")

    @property
    def timings(self):
        return self._timings

    @property
    def session(self):
        return self._s


def acpf_nr_gpu(out, ac_Ybus, V, Sbus, slack_ids, slack_weights, pv, pq, max_iter, tol, nb_solve=1,
                device=-1, precision="fp64"):
    """One AC power flow, written into ``out`` in place (the reference's
    ``acpf_nr_gpu``).  ``nb_solve`` repeats the solve (timing loop); the
    timings of the last one are returned."""
    out_arr = np.asarray(out)
    if out_arr.dtype != np.complex128 or not out_arr.flags.c_contiguous:
        raise ValueError("out must be a C-contiguous complex128 array")
    ac = AcPfGPU((ac_Ybus, V, Sbus, slack_ids, slack_weights, pv, pq), precision=precision,
                 max_iter=max_iter, tol=tol, device=normalize_device(device) if device != -1 else None,
                 init_from_n_powerflow=False)
    for _ in range(max(int(nb_solve), 1) - 1):
        ac.resolve(V)
    out_arr[...] = ac.solve()
    return ac.timings
