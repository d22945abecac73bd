"""Learned warm start: an MLP that predicts each row's solution voltages, so
the Newton loop starts a step or two from convergence instead of from a
flat or base-case start.

The reference's batch facades start rows from the base case or from a
caller-given warm start (``ScenarioSweepGPU``'s per-row V0,
``src/gpusim2grid/scenario_sweep/gpu_facade.py``); this module produces such
a V0 on the GPU, and the sweep converges it with the same FP64 mismatch and
tolerance as any other start, so the prediction changes how many Newton
steps a row takes, never its answer.  A row whose predicted start fails is
restarted from Vinit inside the same kernel launch (``rescue``).

Network: x -> [Linear -> GELU] x layers -> Linear -> y (``hidden`` wide),
trained with Adam on mean-squared error.  Every GEMM runs on the tcgen05
BF16 kernel of ``csrc/mlp_kernels.cu`` (fp32 accumulation), as do the bias,
activation, loss-gradient, bias-gradient, transpose, Adam and
voltage-assembly steps; PyTorch only holds the device buffers and gathers
the minibatches.

Features of a row (``LearnedStart.features``), all per unit:
  [dP at pv+pq buses | dQ at pq buses]      its injections minus the base case
  [oP at pv+pq buses | oQ at pq buses]      the base-case flow of every
                                            tripped branch, put at its two
                                            end buses (the injection that
                                            would replace the branch)
Targets: [Va at pv+pq buses | Vm at pq buses] of the converged row, the
unknowns of the reference's Newton step (``src/_cpp/acpf_nr.cu``); slack
and pv magnitudes come from Vinit.  Inputs and targets are standardised
per column with the training set's statistics.
"""

from __future__ import annotations

import time

import numpy as np
import torch

from ._common import RowStatus, grid_arrays, make_session
from ._native import lib

__all__ = ["WarmStartMLP", "LearnedStart", "make_training_rows", "generate_solutions"]

_M = lib.mlp


def _ceil(x, m):
    return (int(x) + m - 1) // m * m


def _stream():
    return torch.cuda.current_stream().cuda_stream


class WarmStartMLP:
    """BF16 MLP on the tcgen05 GEMM.  ``n_in`` inputs and ``n_out`` outputs
    are padded to multiples of 128 on the device; ``hidden`` is rounded up to
    one.  Master weights are fp32 (Adam updates them), the GEMMs read their
    bf16 copies."""

    def __init__(self, n_in, n_out, hidden=1024, layers=2, device=None, seed=0):
        if layers < 1:
            raise ValueError("layers must be >= 1")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else int(device))
        self.n_in, self.n_out = int(n_in), int(n_out)
        self.k0, self.h, self.o = _ceil(n_in, 128), _ceil(hidden, 128), _ceil(n_out, 128)
        self.layers = int(layers)
        dims = [self.k0] + [self.h] * layers + [self.o]
        self.shapes = [(dims[l + 1], dims[l]) for l in range(layers + 1)]
        # one flat fp32 buffer for weights and biases (Adam runs over it in one
        # launch); every piece starts on a 64-element boundary
        offs, n = [], 0
        for (o, i) in self.shapes:
            offs.append((n, _ceil(n + o * i, 64)))
            n = _ceil(n + o * i, 64) + _ceil(o, 64)
        self._offs, self._n = offs, n
        dev = self.device
        self.master = torch.zeros(n, dtype=torch.float32, device=dev)
        self.grad = torch.zeros_like(self.master)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.wb = torch.zeros(n, dtype=torch.bfloat16, device=dev)
        gen = torch.Generator(device="cpu").manual_seed(int(seed))
        fan_in = [self.n_in] + [self.h] * layers
        for l, (o, i) in enumerate(self.shapes):
            w = torch.randn(o, i, generator=gen) / np.sqrt(fan_in[l])
            if l == 0:
                w[:, self.n_in:] = 0
            if l == layers:
                w[self.n_out:, :] = 0
            self.W(l).copy_(w)
        self.wb.copy_(self.master)
        self.step = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.x_mean = torch.zeros(self.n_in, dtype=torch.float32, device=dev)
        self.x_std = torch.ones(self.n_in, dtype=torch.float32, device=dev)
        self.y_mean = torch.zeros(self.n_out, dtype=torch.float32, device=dev)
        self.y_std = torch.ones(self.n_out, dtype=torch.float32, device=dev)
        self._ws = {}
        self._stats_ver = 0
        self._sparse = (None, None)

    # -------------------------------------------------------------- params
    def _view(self, buf, l, bias):
        o, i = self.shapes[l]
        w0, b0 = self._offs[l]
        return buf[b0:b0 + o] if bias else buf[w0:w0 + o * i].view(o, i)

    def W(self, l):
        return self._view(self.master, l, False)

    def b(self, l):
        return self._view(self.master, l, True)

    def parameters_fp32(self):
        """[(W_l, b_l)] fp32 master copies, W_l (out, in) including padding."""
        return [(self.W(l), self.b(l)) for l in range(self.layers + 1)]

    def set_stats(self, x_mean, x_std, y_mean, y_std, floor=1e-6):
        """Per-column standardisation of inputs and targets.  A std below
        ``floor`` (per unit / radians) is raised to it: such a column is
        constant for the network's purpose (e.g. the voltage of a load-free
        bus fed only from the slack), and dividing by a std at the level of
        solver noise would blow the fp32 rounding of its mean up."""
        f = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float32), device=self.device)
        self.x_mean, self.x_std = f(x_mean), torch.clamp(f(np.nan_to_num(x_std, nan=1.0)), min=floor)
        self.y_mean, self.y_std = f(y_mean), torch.clamp(f(np.nan_to_num(y_std, nan=1.0)), min=floor)
        self._stats_ver += 1

    # ------------------------------------------------------------- buffers
    def device_inputs(self, F):
        """Raw features (rows, n_in) on the device -> standardised bf16
        (rows padded to 128, k0)."""
        r = F.shape[0]
        X = torch.zeros(_ceil(max(r, 1), 128), self.k0, dtype=torch.bfloat16, device=self.device)
        X[:r, :self.n_in] = ((F.to(torch.float32) - self.x_mean) / self.x_std).to(torch.bfloat16)
        return X

    def device_targets(self, Yraw):
        """Raw targets (rows, n_out) -> standardised fp32 (rows padded, o)."""
        r = Yraw.shape[0]
        T = torch.zeros(_ceil(max(r, 1), 128), self.o, dtype=torch.float32, device=self.device)
        T[:r, :self.n_out] = ((Yraw.to(torch.float64) - self.y_mean.double()) / self.y_std.double()).float()
        return T

    def _buffers(self, B, train):
        key = (B, train)
        if key in self._ws:
            return self._ws[key]
        dev, f32, bf = self.device, torch.float32, torch.bfloat16
        L = self.layers
        w = dict(pre=[torch.empty(B, self.h, dtype=f32, device=dev) for _ in range(L)],
                 act=[torch.empty(B, self.h, dtype=bf, device=dev) for _ in range(L)],
                 y=torch.empty(B, self.o, dtype=f32, device=dev))
        if train:
            w.update(dy=torch.empty(B, self.o, dtype=bf, device=dev),
                     g=torch.empty(B, self.h, dtype=bf, device=dev),
                     gT=torch.empty(max(self.h, self.o), B, dtype=bf, device=dev),
                     aT=torch.empty(max(self.h, self.k0), B, dtype=bf, device=dev),
                     WT=torch.empty(self.h, max(self.h, self.o), dtype=bf, device=dev),
                     da=torch.empty(B, self.h, dtype=f32, device=dev),
                     loss=torch.zeros(1, dtype=f32, device=dev))
        self._ws[key] = w
        return w

    # ------------------------------------------------------------- kernels
    def _gemm(self, A, B, D, acc=False):
        M, K = A.shape
        N, K2 = B.shape
        if K != K2 or tuple(D.shape) != (M, N):
            raise ValueError(f"gemm shapes {tuple(A.shape)} x {tuple(B.shape)}^T -> {tuple(D.shape)}")
        _M.gemm_tn_bf16(A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), D.data_ptr(), D.stride(0), M, N, K,
                        acc, self.err.data_ptr(), _stream())

    def _wb(self, l):
        return self._view(self.wb, l, False)

    def _forward(self, X, w):
        self._gemm(X, self._wb(0), w["pre"][0])
        return self._forward_rest(w, X.shape[0])

    def _forward_rest(self, w, B):
        """The network from the first layer's pre-activations w['pre'][0]
        (B rows) to its outputs w['y']."""
        L = self.layers
        for l in range(L + 1):
            if l > 0:
                self._gemm(w["act"][l - 1], self._wb(l), w["pre"][l] if l < L else w["y"])
            if l < L:
                _M.bias_act(w["pre"][l].data_ptr(), self.h, self.b(l).data_ptr(), w["act"][l].data_ptr(), self.h,
                            B, self.h, True, _stream())
            else:
                _M.bias_act(w["y"].data_ptr(), self.o, self.b(l).data_ptr(), 0, self.o, B, self.o, False,
                            _stream())
        return w["y"]

    def _sparse_first(self):
        """(W0T, base) of the current first-layer weights and input
        standardisation: W0^T [k0 x h] bf16 and the first layer's product
        with an all-zero raw input row (gs2g_mlp_first_layer_base); rebuilt
        after a training step or new statistics."""
        key = (self.step, self._stats_ver)
        if self._sparse[0] != key:
            W0 = self._wb(0)
            W0T = torch.empty(self.k0, self.h, dtype=torch.bfloat16, device=self.device)
            _M.transpose_bf16(W0.data_ptr(), W0.stride(0), W0T.data_ptr(), W0T.stride(0), self.h, self.k0, _stream())
            base = torch.empty(self.h, dtype=torch.float32, device=self.device)
            _M.first_layer_base(W0T.data_ptr(), self.h, self.x_mean.data_ptr(), self.x_std.data_ptr(), self.n_in,
                                base.data_ptr(), _stream())
            self._sparse = (key, (W0T, base))
        return self._sparse[1]

    def predict_trips(self, trip_ptr, trip_ids, br_cols, br_vals, n_rows, chunk=16384):
        """Standardised outputs (rows padded to 128, o) fp32 of rows whose raw
        inputs are only their tripped branches' contributions (no injection
        part; device int32 CSR trip_ptr / trip_ids, the per-branch columns
        and values of ``LearnedStart``): the first layer from those few
        columns (gs2g_mlp_sparse_first_layer), the other layers on the GEMM.
        Equals ``predict`` of the same rows' inputs up to the fp32 summation
        order of the first layer."""
        W0T, base = self._sparse_first()
        rp = _ceil(max(int(n_rows), 1), 128)
        out = None
        for r0 in range(0, rp, chunk):
            B = min(chunk, rp - r0)
            w = self._buffers(B, False)
            rows = max(0, min(B, int(n_rows) - r0))
            _M.sparse_first_layer(base.data_ptr(), W0T.data_ptr(), self.h, trip_ptr.data_ptr() + 4 * r0,
                                  trip_ids.data_ptr(), br_cols.data_ptr(), br_vals.data_ptr(), self.x_mean.data_ptr(),
                                  self.x_std.data_ptr(), self.n_in, w["pre"][0].data_ptr(), self.h, rows, B,
                                  _stream())
            y = self._forward_rest(w, B)
            if rp <= chunk:
                return y
            if out is None:
                out = torch.empty(rp, self.o, dtype=torch.float32, device=self.device)
            out[r0:r0 + B].copy_(y)
        return out

    def _backward(self, X, T, w, scale):
        """Gradients of 0.5 * scale * ||y - T||^2 over the valid columns into
        self.grad; accumulates the squared error into w['loss']."""
        B = X.shape[0]
        L = self.layers
        st = _stream()
        _M.mse_grad(w["y"].data_ptr(), T.data_ptr(), self.o, w["dy"].data_ptr(), B, self.o, self.n_out, scale,
                    w["loss"].data_ptr(), st)
        g, gcols = w["dy"], self.o
        for l in range(L, -1, -1):
            o, i = self.shapes[l]
            a = X if l == 0 else w["act"][l - 1]
            gT = w["gT"][:o]
            aT = w["aT"][:i]
            _M.transpose_bf16(g.data_ptr(), g.stride(0), gT.data_ptr(), B, B, o, st)
            _M.transpose_bf16(a.data_ptr(), a.stride(0), aT.data_ptr(), B, B, i, st)
            self._gemm(gT, aT, self._view(self.grad, l, False))
            _M.colsum_bf16(g.data_ptr(), g.stride(0), B, o, self._view(self.grad, l, True).data_ptr(), st)
            if l > 0:
                WT = w["WT"][:i, :o]
                _M.transpose_bf16(self._wb(l).data_ptr(), i, WT.data_ptr(), WT.stride(0), o, i, st)
                self._gemm(g, WT, w["da"])
                _M.gelu_bwd(w["da"].data_ptr(), self.h, w["pre"][l - 1].data_ptr(), self.h, w["g"].data_ptr(),
                            self.h, B, self.h, st)
                g = w["g"]

    def gradients(self, X, T, scale=None):
        """One forward + backward on a batch (X bf16, T fp32, rows a multiple
        of 128).  Returns ([(dW_l, db_l)], loss) as fp32 device tensors.
        Default scale: 2 / (rows * n_out), the mean-squared-error gradient."""
        B = X.shape[0]
        w = self._buffers(B, True)
        scale = 2.0 / (B * self.n_out) if scale is None else float(scale)
        w["loss"].zero_()
        self._forward(X, w)
        self._backward(X, T, w, scale)
        self.check()
        grads = [(self._view(self.grad, l, False).clone(), self._view(self.grad, l, True).clone())
                 for l in range(self.layers + 1)]
        return grads, float(w["loss"].item())

    def check(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a bounded wait in the tcgen05 GEMM ran out; its output is not valid")

    # ------------------------------------------------------------ training
    def fit_device(self, X, T, epochs=20, batch=1024, lr=1e-3, lr_decay=0.8, weight_decay=0.0, seed=0,
                   n_rows=None, X_val=None, T_val=None, n_val=None):
        """Adam on device-resident standardised data (``device_inputs`` /
        ``device_targets``).  ``n_rows``: valid rows of X/T (default all).
        One learning rate per epoch, multiplied by ``lr_decay`` after each.
        Returns {'loss': [...], 'val': [...]} (mean squared error per valid
        entry, in standardised units)."""
        n = X.shape[0] if n_rows is None else int(n_rows)
        B = _ceil(min(batch, max(n, 128)), 128)
        nb = n // B
        if nb < 1:
            raise ValueError(f"need at least one batch of {B} rows, have {n}")
        w = self._buffers(B, True)
        gen = torch.Generator(device=self.device).manual_seed(int(seed))
        hist, val = [], []
        scale = 2.0 / (B * self.n_out)
        cur = float(lr)
        for ep in range(int(epochs)):
            perm = torch.randperm(n, generator=gen, device=self.device)
            w["loss"].zero_()
            for i in range(nb):
                idx = perm[i * B:(i + 1) * B]
                Xb = X.index_select(0, idx)
                Tb = T.index_select(0, idx)
                self._forward(Xb, w)
                self._backward(Xb, Tb, w, scale)
                self.step += 1
                _M.adam(self.master.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                        self.wb.data_ptr(), self._n, cur, 0.9, 0.999, 1e-8, self.step, float(weight_decay),
                        _stream())
            hist.append(w["loss"])
            w["loss"] = torch.zeros(1, dtype=torch.float32, device=self.device)
            if X_val is not None:
                val.append(self.mse(X_val, T_val, n_val))
            cur *= float(lr_decay)
        self.check()
        denom = nb * B * self.n_out
        return {"loss": [float(h.item()) / denom for h in hist], "val": val}

    def mse(self, X, T, n_rows=None):
        """Mean squared error per valid entry on standardised data."""
        n = X.shape[0] if n_rows is None else int(n_rows)
        y = self.predict(X)
        d = (y[:n, :self.n_out] - T[:n, :self.n_out]).double()
        return float((d * d).mean().item())

    # ----------------------------------------------------------- inference
    def predict(self, X, chunk=16384):
        """Standardised outputs (rows, o) fp32 for standardised bf16 inputs.
        Up to ``chunk`` rows the result is the network's own output buffer,
        reused by the next call of the same size."""
        R = X.shape[0]
        if R <= chunk:
            return self._forward(X, self._buffers(R, False))
        out = torch.empty(R, self.o, dtype=torch.float32, device=self.device)
        for r0 in range(0, R, chunk):
            Xc = X[r0:r0 + chunk]
            w = self._buffers(Xc.shape[0], False)
            out[r0:r0 + Xc.shape[0]].copy_(self._forward(Xc, w))
        return out


# ---------------------------------------------------------------- grid side
def make_training_rows(grid, n_rows, seed=0, p_outage=0.9, broad=0.5, local_sigma=0.03):
    """Synthetic operating points for training: every row scales the loads
    (a ``broad`` share of rows: global U(0.8, 1.2) x per-bus lognormal(0, 0.1),
    the spread of ``synthetic.injection_scenarios``; the rest: per-bus
    lognormal(0, local_sigma) around the base case), rebalances generation,
    and with probability ``p_outage`` trips one branch whose loss keeps the
    grid connected.  Returns (p_mw, q_mvar, trips)."""
    from .synthetic import n1_branches
    rng = np.random.default_rng(seed)
    n = int(n_rows)
    nl = grid.load_bus.size
    g = np.where(rng.random((n, 1)) < broad, rng.uniform(0.8, 1.2, (n, 1)), 1.0)
    sig = np.where(rng.random((n, 1)) < broad, 0.1, local_sigma)
    scale = g * np.exp(sig * rng.standard_normal((n, nl)))
    lp = grid.load_p[None, :] * scale
    lq = grid.load_q[None, :] * scale
    gp = grid.gen_p[None, :] * (lp.sum(axis=1, keepdims=True) / grid.load_p.sum())
    p = np.zeros((n, grid.n_bus))
    q = np.zeros((n, grid.n_bus))
    np.add.at(p, (slice(None), grid.gen_bus), gp)
    np.subtract.at(p, (slice(None), grid.load_bus), lp)
    np.subtract.at(q, (slice(None), grid.load_bus), lq)
    cand = n1_branches(grid)
    out = rng.random(n) < p_outage
    pick = rng.integers(0, cand.size, n)
    trips = [[int(cand[pick[r]])] if out[r] else [] for r in range(n)]
    return p * grid.sn_mva, q * grid.sn_mva, trips


def _csr(trips):
    ptr = np.zeros(len(trips) + 1, dtype=np.int32)
    ptr[1:] = np.cumsum([len(t) for t in trips])
    ids = np.fromiter((b for t in trips for b in t), dtype=np.int32, count=int(ptr[-1]))
    return ptr, ids


def generate_solutions(grid, p_mw, q_mvar, trips, device=None, chunk=16384, max_iter=30, tol=1e-10):
    """Solve training rows with the GPU sweep (FP64 LU, continuous schedule,
    from the base case).  Returns (V, ok): V (rows, n_bus) complex128 on the
    device, ok (rows,) bool, True where the row converged."""
    d = grid_arrays(grid.as_tuple())
    s = make_session(d, device)
    _base_voltage(s, d)  # kept by the session as the rows' start
    s.set_branch_data(*_branch_arrays(grid))
    n = p_mw.shape[0]
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    V = torch.empty(n, d["n_bus"], dtype=torch.complex128, device=dev)
    ok = torch.empty(n, dtype=torch.bool, device=dev)
    for r0 in range(0, n, chunk):
        r1 = min(n, r0 + chunk)
        s.set_injections(np.ascontiguousarray(p_mw[r0:r1]), np.ascontiguousarray(q_mvar[r0:r1]), grid.sn_mva)
        s.set_contingencies(*_csr(trips[r0:r1]))
        s.run(max_iter, tol, False, lib.PREC_FP64, lib.START_BASE, 0.0, 0, False, 0)
        V[r0:r1] = torch.from_dlpack(s.dlpack("v"))
        ok[r0:r1] = torch.from_dlpack(s.dlpack("status")) == int(RowStatus.CONVERGED)
    torch.cuda.synchronize(dev)
    s.close()
    return V, ok


def _branch_arrays(grid):
    c = lambda a: np.ascontiguousarray(a, dtype=np.complex128)
    return (np.ascontiguousarray(grid.branch_from, dtype=np.int32),
            np.ascontiguousarray(grid.branch_to, dtype=np.int32), c(grid.yff), c(grid.yft), c(grid.ytf),
            c(grid.ytt))


def _base_voltage(s, d, max_iter=20, tol=1e-10):
    V, st, it, res = s.solve_base(max_iter, tol, lib.PREC_FP64, 0.0)
    if st != RowStatus.CONVERGED:
        raise RuntimeError(f"the base case did not converge (residual {res:.3e})")
    return V


class LearnedStart:
    """Learned start voltages for the rows of one grid.

    ``grid`` is the synthetic ``Grid`` (array tuple + branch data).  ``train``
    generates and solves training rows on the GPU and fits the network;
    ``start_voltages`` turns row definitions (injections, tripped branches)
    into V0 on the device.  ``sparse_first_layer`` (default on): rows
    without injection part take the network's first layer from the few input
    columns their tripped branches reach (``WarmStartMLP.predict_trips``)
    instead of the dense input block and its GEMM."""

    def __init__(self, grid, hidden=1024, layers=2, device=None, seed=0):
        self.grid = grid
        self.sparse_first_layer = True
        d = grid_arrays(grid.as_tuple())
        self._d = d
        n = d["n_bus"]
        pv, pq = d["pv"], d["pq"]
        pvpq = np.concatenate([pv, pq])
        self.n_pvpq, self.n_pq = pvpq.size, pq.size
        self.dim = pvpq.size + pq.size
        ia = np.full(n, -1, dtype=np.int32)
        ia[pvpq] = np.arange(pvpq.size, dtype=np.int32)
        im = np.full(n, -1, dtype=np.int32)
        im[pq] = pvpq.size + np.arange(pq.size, dtype=np.int32)
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        dev = self.device
        self._pvpq = torch.as_tensor(pvpq.astype(np.int64), device=dev)
        self._pq = torch.as_tensor(pq.astype(np.int64), device=dev)
        self._ia = torch.as_tensor(ia, device=dev)
        self._im = torch.as_tensor(im, device=dev)
        self._vinit = torch.as_tensor(d["Vinit"], device=dev)
        self._sbase = torch.as_tensor(d["Sbus"], device=dev)
        # base case and the equivalent injection of every branch
        s = make_session(d, device)
        Vb = _base_voltage(s, d)
        s.close()
        self.V_base = Vb
        f, t = grid.branch_from.astype(np.int64), grid.branch_to.astype(np.int64)
        # an open end (negative endpoint) has V = 0 and carries no power
        hf, ht = f >= 0, t >= 0
        fz, tz = np.where(hf, f, 0), np.where(ht, t, 0)
        Vf, Vt = np.where(hf, Vb[fz], 0), np.where(ht, Vb[tz], 0)
        Sft = np.where(hf, Vf * np.conj(grid.yff * Vf + grid.yft * Vt), 0)
        Stf = np.where(ht, Vt * np.conj(grid.ytf * Vf + grid.ytt * Vt), 0)
        off = self.dim  # outage channel
        scratch = 2 * self.dim  # column for entries at the slack / pv Q / an open end (dropped)
        col = lambda m, b, base: np.where((b >= 0) & (m[np.maximum(b, 0)] >= 0), base + m[np.maximum(b, 0)], scratch)
        cols = np.stack([col(ia, f, off), col(im, f, off), col(ia, t, off), col(im, t, off)], axis=1)
        vals = np.stack([Sft.real, Sft.imag, Stf.real, Stf.imag], axis=1)
        self._br_cols = torch.as_tensor(cols.astype(np.int64), device=dev)
        self._br_vals = torch.as_tensor(vals.astype(np.float32), device=dev)
        # the same tables for the fused input kernel (int32; the scratch
        # column n_in is dropped by the kernel)
        self._pvpq32 = self._pvpq.to(torch.int32)
        self._pq32 = self._pq.to(torch.int32)
        self._br_cols32 = self._br_cols.to(torch.int32).contiguous()
        self._br_vals32 = self._br_vals.contiguous()
        self._trips_dev = (None, None)
        self._xbuf = {}
        self.n_in = 2 * self.dim
        self.net = WarmStartMLP(self.n_in, self.dim, hidden=hidden, layers=layers, device=self.device.index,
                                seed=seed)
        self.report = {}

    # ------------------------------------------------------------ features
    def features(self, sbus_rows=None, trips=None, n_rows=None):
        """Raw features (rows, n_in) fp32 on the device.  ``sbus_rows``:
        (rows, n_bus) complex per unit (device tensor or array; None: base
        injections).  ``trips``: list of tripped-branch lists or a CSR
        (ptr, ids) pair of arrays or device tensors (None: no trips)."""
        if n_rows is None:
            n_rows = sbus_rows.shape[0] if sbus_rows is not None else (
                len(trips[0]) - 1 if isinstance(trips, tuple) else len(trips))
        F = torch.zeros(n_rows, self.n_in + 1, dtype=torch.float32, device=self.device)
        if sbus_rows is not None:
            S = torch.as_tensor(sbus_rows, device=self.device)
            dS = S - self._sbase
            F[:, :self.n_pvpq] = dS.real.index_select(1, self._pvpq).float()
            F[:, self.n_pvpq:self.dim] = dS.imag.index_select(1, self._pq).float()
        if trips is not None:
            ptr, ids = trips if isinstance(trips, tuple) else _csr(trips)
            if len(ids):
                if isinstance(ptr, torch.Tensor):  # device CSR (e.g. a session's own row definitions)
                    pt = ptr.to(device=self.device, dtype=torch.int64)
                    r = torch.repeat_interleave(torch.arange(n_rows, device=self.device), pt[1:] - pt[:-1],
                                                output_size=len(ids))
                    b = ids.to(device=self.device, dtype=torch.int64)
                else:
                    rows = np.repeat(np.arange(n_rows, dtype=np.int64), np.diff(ptr))
                    r = torch.as_tensor(rows, device=self.device)
                    b = torch.as_tensor(np.asarray(ids, dtype=np.int64), device=self.device)
                cols = self._br_cols.index_select(0, b)
                vals = self._br_vals.index_select(0, b)
                F.index_put_((r[:, None].expand(-1, 4), cols), vals, accumulate=True)
        return F[:, :self.n_in]

    def targets(self, V):
        """(rows, dim) FP64 unknowns [Va at pv+pq | Vm at pq] of voltages V."""
        V = torch.as_tensor(V, device=self.device)
        return torch.cat([torch.angle(V).index_select(1, self._pvpq), torch.abs(V).index_select(1, self._pq)], 1)

    # ------------------------------------------------------------ training
    def train(self, n_rows=100000, epochs=20, batch=1024, lr=1e-3, lr_decay=0.8, seed=0, val_fraction=0.02,
              **row_kw):
        """Generate ``n_rows`` operating points, solve them on the GPU, fit the
        network.  Returns a report dict (times in seconds, losses)."""
        t0 = time.perf_counter()
        p, q, trips = make_training_rows(self.grid, n_rows, seed=seed, **row_kw)
        t1 = time.perf_counter()
        V, ok = generate_solutions(self.grid, p, q, trips, device=self.device.index)
        t2 = time.perf_counter()
        keep = ok.nonzero().flatten()
        sb = torch.as_tensor((p + 1j * q) / self.grid.sn_mva, device=self.device)
        F = self.features(sb, trips).index_select(0, keep)
        Yt = self.targets(V).index_select(0, keep)
        nk = int(keep.numel())
        x_mean, x_std = F.mean(0), F.std(0)
        y_mean, y_std = Yt.mean(0), Yt.std(0)
        self.net.set_stats(x_mean.cpu().numpy(), x_std.cpu().numpy(), y_mean.cpu().numpy(), y_std.cpu().numpy())
        n_val = int(nk * val_fraction) // 128 * 128  # predict() takes whole 128-row tiles
        X = self.net.device_inputs(F)
        T = self.net.device_targets(Yt)
        n_tr = nk - n_val
        Xv = Tv = None
        if n_val:
            Xv, Tv = X[n_tr:n_tr + n_val].contiguous(), T[n_tr:n_tr + n_val].contiguous()
        torch.cuda.synchronize(self.device)
        t3 = time.perf_counter()
        hist = self.net.fit_device(X, T, epochs=epochs, batch=batch, lr=lr, lr_decay=lr_decay, seed=seed,
                                   n_rows=n_tr, X_val=Xv, T_val=Tv, n_val=n_val)
        torch.cuda.synchronize(self.device)
        t4 = time.perf_counter()
        self.report = dict(n_rows=n_rows, n_train=n_tr, n_val=n_val, n_unconverged=n_rows - nk,
                           t_rows_s=t1 - t0, t_solve_s=t2 - t1, t_features_s=t3 - t2, t_fit_s=t4 - t3,
                           loss=hist["loss"], val=hist["val"])
        return self.report

    # ----------------------------------------------------------- inference
    def _device_trips(self, trips):
        """(ptr, ids) int32 device tensors of a trip CSR given as device
        tensors, arrays or a list of lists (the last conversion is kept)."""
        if trips is None:
            return None, None
        key = trips if isinstance(trips, tuple) else None
        if key is not None and self._trips_dev[0] is key:
            return self._trips_dev[1]
        ptr, ids = trips if isinstance(trips, tuple) else _csr(trips)
        cv = lambda a: torch.as_tensor(a if isinstance(a, torch.Tensor) else np.asarray(a),
                                       device=self.device).to(torch.int32).contiguous()
        out = (cv(ptr), cv(ids) if len(ids) else torch.zeros(1, dtype=torch.int32, device=self.device))
        self._trips_dev = (key, out)
        return out

    def inputs(self, sbus_rows=None, trips=None, n_rows=None):
        """Standardised bf16 network inputs (rows padded to 128, k0) in one
        fused kernel (gs2g_mlp_features): the same values as
        ``net.device_inputs(features(...))``, without the intermediate
        tensors.  The returned block is reused by the next call."""
        if n_rows is None:
            n_rows = sbus_rows.shape[0] if sbus_rows is not None else (
                len(trips[0]) - 1 if isinstance(trips, tuple) else len(trips))
        net = self.net
        rp = _ceil(max(n_rows, 1), 128)
        X = self._xbuf.get(rp)
        if X is None:
            X = self._xbuf[rp] = torch.empty(rp, net.k0, dtype=torch.bfloat16, device=self.device)
        sb = None
        if sbus_rows is not None:
            sb = torch.as_tensor(sbus_rows, device=self.device)
            if sb.dtype != torch.complex128 or not sb.is_contiguous():
                sb = sb.to(torch.complex128).contiguous()
        tp, ti = self._device_trips(trips)
        _M.features(0 if sb is None else sb.data_ptr(), self._sbase.data_ptr(), self._pvpq32.data_ptr(), self.n_pvpq,
                    self._pq32.data_ptr(), self.n_pq, 0 if tp is None else tp.data_ptr(),
                    0 if ti is None else ti.data_ptr(), self._br_cols32.data_ptr(), self._br_vals32.data_ptr(),
                    net.x_mean.data_ptr(), net.x_std.data_ptr(), net.n_in, X.data_ptr(), net.k0, n_rows, rp,
                    self._d["n_bus"], _stream())
        return X, n_rows

    def start_voltages(self, sbus_rows=None, trips=None, n_rows=None, out_ptr=None):
        """Predicted V0 (rows, n_bus) complex128 on the device, enqueued on
        torch's current stream.  With ``out_ptr`` (a device address of rows x
        n_bus complex128, e.g. a session's ``start_rows_buffer``) V0 is
        written there and None is returned."""
        if sbus_rows is None and trips is not None and self.sparse_first_layer:
            # outage rows at the base injections: the first layer from the
            # few input columns their tripped branches reach
            R = int(n_rows) if n_rows is not None else (
                len(trips[0]) - 1 if isinstance(trips, tuple) else len(trips))
            tp, ti = self._device_trips(trips)
            y = self.net.predict_trips(tp, ti, self._br_cols32, self._br_vals32, R)
        else:
            X, R = self.inputs(sbus_rows, trips, n_rows)
            y = self.net.predict(X)
        V0 = None
        if out_ptr is None:
            V0 = torch.empty(R, self._d["n_bus"], dtype=torch.complex128, device=self.device)
            out_ptr = V0.data_ptr()
        _M.start_voltages(y.data_ptr(), self.net.o, self.net.y_mean.data_ptr(), self.net.y_std.data_ptr(),
                          self._ia.data_ptr(), self._im.data_ptr(), self._vinit.data_ptr(), self._d["n_bus"],
                          int(out_ptr), R, _stream())
        return V0

    def launches_per_call(self, n_rows, sbus_rows=True):
        """Kernels of this library one ``start_voltages`` call launches: the
        fused inputs, a GEMM and a bias/activation per layer and chunk, the
        start voltages; without injection rows (``sbus_rows`` False) the
        first layer's sparse product (per chunk) replaces the inputs and the
        first GEMM."""
        chunks = max(1, -(-_ceil(max(n_rows, 1), 128) // 16384))
        if not sbus_rows and self.sparse_first_layer:
            return (2 * self.net.layers + 2) * chunks + 1
        return 2 * (self.net.layers + 1) * chunks + 2
