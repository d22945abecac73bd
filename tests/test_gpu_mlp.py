"""The warm-start MLP's device routines against FP64 math: the tcgen05 BF16
GEMM, and one forward + backward of the network against the CPU oracle
(oracle/mlp_oracle.py) with the same bf16 rounding points."""

import numpy as np
import pytest

from oracle import mlp_oracle as MO

pytestmark = pytest.mark.gpu


def _bf16(t):
    import torch
    return t.to(torch.bfloat16)


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 1216), (1024, 1024, 7232)])
def test_gemm_tn_bf16_matches_fp64(M, N, K):
    import torch
    from gpusim2grid_b200._native import lib
    g = torch.Generator().manual_seed(M + N + K)
    A = _bf16(torch.randn(M, K, generator=g)).cuda()
    B = _bf16(torch.randn(N, K, generator=g)).cuda()
    D = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    lib.mlp.gemm_tn_bf16(A.data_ptr(), K, B.data_ptr(), K, D.data_ptr(), N, M, N, K, False, err.data_ptr(), s)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.double().cpu().numpy() @ B.double().cpu().numpy().T
    got = D.cpu().numpy()
    # exact bf16 products, fp32 accumulation over K terms of size ~1
    tol = 1e-5 * np.sqrt(K) * np.abs(ref).max() + 1e-5
    assert np.abs(got - ref).max() < tol
    # accumulate mode adds to D
    lib.mlp.gemm_tn_bf16(A.data_ptr(), K, B.data_ptr(), K, D.data_ptr(), N, M, N, K, True, err.data_ptr(), s)
    torch.cuda.synchronize()
    assert np.abs(D.cpu().numpy() - 2 * ref).max() < 2 * tol


def test_gemm_rejects_bad_shapes():
    import torch
    from gpusim2grid_b200._native import lib
    A = torch.zeros(100, 64, dtype=torch.bfloat16, device="cuda")
    D = torch.zeros(100, 128, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(ValueError):
        lib.mlp.gemm_tn_bf16(A.data_ptr(), 64, A.data_ptr(), 64, D.data_ptr(), 128, 100, 128, 64, False,
                             err.data_ptr(), 0)


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.parametrize("layers", [1, 2])
def test_forward_backward_match_oracle(layers):
    import torch
    from gpusim2grid_b200.warmstart import WarmStartMLP
    n_in, n_out, B = 300, 150, 256
    net = WarmStartMLP(n_in, n_out, hidden=256, layers=layers, seed=3)
    rng = np.random.default_rng(5)
    Xr = rng.standard_normal((B, n_in)).astype(np.float32)
    Tr = rng.standard_normal((B, n_out)).astype(np.float32)
    X = net.device_inputs(torch.as_tensor(Xr, device="cuda"))
    T = net.device_targets(torch.as_tensor(Tr, device="cuda"))
    grads, loss = net.gradients(X, T)
    y = net.predict(X).cpu().numpy()

    Ws = [W.cpu().numpy().astype(np.float64) for W, _ in net.parameters_fp32()]
    bs = [b.cpu().numpy().astype(np.float64) for _, b in net.parameters_fp32()]
    Xp = X.float().cpu().numpy()
    Tp = T.cpu().numpy().astype(np.float64)
    scale = 2.0 / (B * n_out)
    y_ref, cache = MO.forward(Ws, bs, Xp, emulate_device=True)
    assert _rel(y[:, :n_out], y_ref[:, :n_out]) < 2e-3
    assert abs(loss - MO.mse_loss(y_ref, Tp, n_out)) < 2e-3 * MO.mse_loss(y_ref, Tp, n_out)
    dWs, dbs = MO.backward(Ws, bs, cache, y_ref, Tp, n_out, scale, emulate_device=True)
    for l, (dW, db) in enumerate(grads):
        assert _rel(dW.cpu().numpy(), dWs[l]) < 1e-2, l
        assert _rel(db.cpu().numpy(), dbs[l]) < 1e-2, l
    # and against plain FP64 math (no bf16 rounding): bf16 operand error
    y64, c64 = MO.forward(Ws, bs, Xp, emulate_device=False)
    dW64, _ = MO.backward(Ws, bs, c64, y64, Tp, n_out, scale, emulate_device=False)
    for l, (dW, _) in enumerate(grads):
        assert _rel(dW.cpu().numpy(), dW64[l]) < 3e-2, l


def test_fit_matches_a_torch_fp32_reference_fit():
    """Training on the device (BF16 GEMMs, fp32 master weights, Adam) ends
    where plain PyTorch fp32 training from the same initial weights with the
    same schedule ends."""
    import torch
    from gpusim2grid_b200.warmstart import WarmStartMLP
    rng = np.random.default_rng(0)
    n, n_in, n_out, hid = 8192, 64, 32, 256
    A = rng.standard_normal((n_in, n_out)) / np.sqrt(n_in)
    Xr = rng.standard_normal((n, n_in))
    Yr = np.tanh(Xr @ A) + 0.1 * (Xr @ A) ** 2
    net = WarmStartMLP(n_in, n_out, hidden=hid, layers=2, seed=1)
    net.set_stats(Xr.mean(0), Xr.std(0), Yr.mean(0), Yr.std(0))
    init = [(W.cpu().clone(), b.cpu().clone()) for W, b in net.parameters_fp32()]
    X = net.device_inputs(torch.as_tensor(Xr, device="cuda"))
    T = net.device_targets(torch.as_tensor(Yr, device="cuda"))
    h = net.fit_device(X, T, epochs=8, batch=512, lr=2e-3, lr_decay=0.8, n_rows=n)
    ours = net.mse(X, T, n)
    assert h["loss"][-1] < 0.25 * h["loss"][0]

    # the same network and schedule in plain PyTorch fp32 on the CPU
    torch.manual_seed(0)
    dims = [(hid, n_in), (hid, hid), (n_out, hid)]
    ref = torch.nn.Sequential(torch.nn.Linear(n_in, hid), torch.nn.GELU(), torch.nn.Linear(hid, hid),
                              torch.nn.GELU(), torch.nn.Linear(hid, n_out))
    lin = [m for m in ref if isinstance(m, torch.nn.Linear)]
    with torch.no_grad():
        for m, (W, b), (o, i) in zip(lin, init, dims):
            m.weight.copy_(W[:o, :i])
            m.bias.copy_(b[:o])
    Xc = torch.tensor((Xr - Xr.mean(0)) / Xr.std(0), dtype=torch.float32)
    Tc = torch.tensor((Yr - Yr.mean(0)) / Yr.std(0), dtype=torch.float32)
    opt = torch.optim.Adam(ref.parameters(), lr=2e-3)
    sch = torch.optim.lr_scheduler.ExponentialLR(opt, 0.8)
    for _ in range(8):
        perm = torch.randperm(n)
        for i in range(n // 512):
            idx = perm[i * 512:(i + 1) * 512]
            loss = ((ref(Xc[idx]) - Tc[idx]) ** 2).mean()
            opt.zero_grad()
            loss.backward()
            opt.step()
        sch.step()
    with torch.no_grad():
        theirs = float(((ref(Xc) - Tc) ** 2).mean())
    assert abs(ours - theirs) < 0.2 * theirs + 0.01, (ours, theirs)


def test_fused_inputs_equal_the_torch_path(g118):
    """gs2g_mlp_features (one kernel: injections, outage contributions,
    standardisation, bf16, padding) against the same inputs built from
    torch ops (features() then device_inputs()), for injection rows with
    one or two trips each and for trip-only rows."""
    import torch
    from gpusim2grid_b200.synthetic import injection_scenarios, n1_branches
    from gpusim2grid_b200.warmstart import LearnedStart
    ls = LearnedStart(g118, hidden=128, layers=1, seed=0)
    rng = np.random.default_rng(4)
    ls.net.set_stats(rng.standard_normal(ls.n_in), rng.uniform(0.5, 2.0, ls.n_in), np.zeros(ls.dim), np.ones(ls.dim))
    p, q = injection_scenarios(g118, 37, seed=3)
    sb = torch.as_tensor((p + 1j * q) / g118.sn_mva, device="cuda")
    cand = n1_branches(g118)
    trips = [[int(cand[r % cand.size])] + ([int(cand[(3 * r) % cand.size])] if r % 3 == 0 else []) for r in range(37)]
    for s_rows, t_rows in ((sb, trips), (None, trips), (sb, None)):
        ref = ls.net.device_inputs(ls.features(s_rows, t_rows, 37))
        X, n = ls.inputs(s_rows, t_rows, 37)
        assert n == 37 and X.shape == ref.shape
        a, b = X.float(), ref.float()
        # equal up to the fp32 summation order of two trips at one bus (one bf16 step at most)
        assert torch.all((a - b).abs() <= 2 ** -7 * b.abs().clamp(min=1e-3))
        assert torch.all(X[37:] == 0) and torch.all(X[:, ls.n_in:] == 0)
