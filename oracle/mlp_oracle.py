"""CPU oracle of the warm-start MLP (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module, and there only as the checker: the product path
(``gpusim2grid_b200.warmstart``) runs the network on the GPU kernels of
``gpusim2grid_b200/csrc/mlp_kernels.cu`` and never calls this file.

The reference has no learned start (its ScenarioSweepGPU accepts any per-row
warm-start voltage, ``src/gpusim2grid/scenario_sweep/gpu_facade.py``), so
there is no reference output to pin this oracle to: it is pinned by its own
finite-difference test (``tests/test_oracle.py``) and checks the device
network, which must agree with it within the bf16 tolerances of the tests.

Network: x -> [Linear -> GELU(erf)] x L -> Linear -> y, mean-squared error
over the first ``n_out`` output columns.  Weights are stored W[out, in].
``forward``/``backward`` with ``emulate_device=True`` round to bf16 at the
same points as the device path does (GEMM operands: inputs, weights,
activations, output gradients, hidden-layer pre-activation gradients), and
compute everything else in FP64; with ``emulate_device=False`` they are
plain FP64 math.
"""

from __future__ import annotations

import numpy as np
from scipy.special import erf

__all__ = ["bf16_round", "gelu", "gelu_grad", "forward", "backward", "mse_loss"]


def bf16_round(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned
    as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    cdf = 0.5 * (1.0 + erf(x / np.sqrt(2.0)))
    pdf = np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)
    return cdf + x * pdf


def _q(x, on):
    return bf16_round(x) if on else np.asarray(x, dtype=np.float64)


def forward(Ws, bs, X, emulate_device=True):
    """Ws[l]: (out, in) weights, bs[l]: (out,) biases; X: (rows, in).
    Returns (y, cache) with y (rows, out_last) in FP64."""
    q = emulate_device
    a = _q(X, q)
    pres, acts = [], [a]
    for l, (W, b) in enumerate(zip(Ws, bs)):
        z = a @ _q(W, q).T + np.asarray(b, dtype=np.float64)
        if l + 1 < len(Ws):
            pres.append(z)
            a = _q(gelu(z), q)
            acts.append(a)
        else:
            y = z
    return y, (pres, acts)


def mse_loss(y, T, n_out):
    d = y[:, :n_out] - np.asarray(T, dtype=np.float64)[:, :n_out]
    return float(np.sum(d * d))


def backward(Ws, bs, cache, y, T, n_out, scale, emulate_device=True):
    """Gradients of 0.5 * scale * sum((y - T)^2) over the first n_out columns
    (the device's dy = scale * (y - T)).  Returns (dWs, dbs)."""
    q = emulate_device
    pres, acts = cache
    dy = np.zeros_like(y)
    dy[:, :n_out] = scale * (y[:, :n_out] - np.asarray(T, dtype=np.float64)[:, :n_out])
    g = _q(dy, q)
    L = len(Ws)
    dWs, dbs = [None] * L, [None] * L
    for l in range(L - 1, -1, -1):
        dWs[l] = g.T @ acts[l]
        dbs[l] = g.sum(axis=0)
        if l > 0:
            da = g @ _q(Ws[l], q)
            g = _q(da * gelu_grad(pres[l - 1]), q)
    return dWs, dbs
