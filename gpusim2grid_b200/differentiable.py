"""Differentiable batched power flow: voltages as a torch function of the
per-row injections, gradients by the batched adjoint.

The reference's ``gpusim2grid.differentiable`` (``BatchPowerFlow``,
``src/gpusim2grid/differentiable/_batch_pf.py``) differentiates a scenario
sweep through its converged state: with F(x, s) = S_calc(x) - s = 0 at the
solution, dx/ds = J^-1, so a loss L(V(x)) has dL/ds = J^-T dL/dx, one
transposed solve per row with the row's Jacobian
(``src/_cpp/contingency/batch_pf_driver.cuh:180-224``).  Here the forward is a
sweep of ``InjectionSweepGPU`` / ``ScenarioSweepGPU`` and the backward
``solve_JT`` (``gs2g_solve_jt``).  Array-tuple mode: the inputs are bus
injections in MW / MVAr (``set_injections``); P at the slack and Q at PV and
slack buses do not change the solution and get zero gradient.
"""

from __future__ import annotations

import numpy as np
import torch

__all__ = ["BatchPowerFlowFunction", "batch_power_flow"]


class BatchPowerFlowFunction(torch.autograd.Function):
    """V = f(P, Q) for the rows of ``sweep`` (a ``InjectionSweepGPU`` or
    ``ScenarioSweepGPU`` with its topology already set).  P, Q: (rows, n_bus)
    float64 in MW / MVAr; V: (rows, n_bus) complex128 on the sweep's device.
    Rows that do not converge give NaN voltages and zero gradients."""

    @staticmethod
    def forward(ctx, p_mw, q_mvar, sweep, sn_mva):
        sweep.set_injections(p_mw.detach().cpu().numpy(), q_mvar.detach().cpu().numpy(), sn_mva)
        sweep.compute()
        dev = torch.device("cuda", sweep._device_index())
        V = torch.from_dlpack(sweep.session.dlpack("v")).clone()
        st = torch.from_dlpack(sweep.session.dlpack("status")).clone()
        V[st != 0] = complex("nan+nanj")
        ctx.sweep = sweep
        ctx.sn_mva = float(sn_mva)
        ctx.save_for_backward(V, st)
        ctx.layout = _layout(sweep, dev)
        return V

    @staticmethod
    def backward(ctx, grad_V):
        V, st = ctx.saved_tensors
        pvpq, pq = ctx.layout
        ok = (st == 0)[:, None]
        g = torch.where(ok, grad_V, torch.zeros_like(grad_V))
        Vs = torch.where(ok, V, torch.ones_like(V))
        # torch's gradient of a real loss w.r.t. complex V is dL/dRe + j dL/dIm;
        # V = Vm e^{j theta}: dL/dtheta = Re(conj(g) j V), dL/dVm = Re(conj(g) V / |V|)
        dth = (g.conj() * 1j * Vs).real
        dvm = (g.conj() * Vs / Vs.abs()).real
        dx = torch.cat([dth[:, pvpq], dvm[:, pq]], dim=1)
        lam = ctx.sweep.solve_JT(dx)  # dL/ds = J^-T dL/dx
        n, nb = V.shape
        gp = torch.zeros((n, nb), dtype=torch.float64, device=V.device)
        gq = torch.zeros_like(gp)
        npvpq = pvpq.numel()
        gp[:, pvpq] = lam[:, :npvpq] / ctx.sn_mva
        gq[:, pq] = lam[:, npvpq:] / ctx.sn_mva
        return gp, gq, None, None


def _layout(sweep, dev):
    d = sweep._d
    pv = np.asarray(d["pv"], dtype=np.int64)
    pq = np.asarray(d["pq"], dtype=np.int64)
    pvpq = np.sort(np.concatenate([pv, pq]))
    return torch.as_tensor(pvpq, device=dev), torch.as_tensor(pq, device=dev)


def batch_power_flow(p_mw, q_mvar, sweep, sn_mva=100.0):
    """Functional form of :class:`BatchPowerFlowFunction`."""
    return BatchPowerFlowFunction.apply(p_mw, q_mvar, sweep, sn_mva)
