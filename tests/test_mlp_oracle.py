"""CPU checks of the MLP oracle: its FP64 backward pass against finite
differences of its loss, and its bf16 rounding against known values."""

import numpy as np

from oracle import mlp_oracle as MO


def test_bf16_round_known_values():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], dtype=np.float32)
    r = MO.bf16_round(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0);
    # 1 + 3 * 2^-8 is a tie between 1 + 2^-7 and 1 + 2^-6: rounds to 1 + 2^-6
    np.testing.assert_array_equal(r[:4], [1.0, 1.0, 1.0 + 2 ** -6, -2.5])
    assert abs(r[4] - 3.0e-3) < 3.0e-3 * 2 ** -8


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    n_in, h, n_out, B = 7, 6, 5, 9
    Ws = [rng.standard_normal((h, n_in)) * 0.5, rng.standard_normal((h, h)) * 0.5,
          rng.standard_normal((n_out + 2, h)) * 0.5]
    bs = [rng.standard_normal(h) * 0.1, rng.standard_normal(h) * 0.1, rng.standard_normal(n_out + 2) * 0.1]
    X = rng.standard_normal((B, n_in))
    T = rng.standard_normal((B, n_out + 2))
    scale = 0.7

    def loss(Ws_, bs_):
        y, _ = MO.forward(Ws_, bs_, X, emulate_device=False)
        return 0.5 * scale * MO.mse_loss(y, T, n_out)

    y, cache = MO.forward(Ws, bs, X, emulate_device=False)
    dWs, dbs = MO.backward(Ws, bs, cache, y, T, n_out, scale, emulate_device=False)
    eps = 1e-6
    for l in range(3):
        for (i, j) in [(0, 0), (1, 2), (Ws[l].shape[0] - 1, Ws[l].shape[1] - 1)]:
            Wp = [w.copy() for w in Ws]
            Wm = [w.copy() for w in Ws]
            Wp[l][i, j] += eps
            Wm[l][i, j] -= eps
            fd = (loss(Wp, bs) - loss(Wm, bs)) / (2 * eps)
            assert abs(fd - dWs[l][i, j]) < 1e-6 * max(1.0, abs(fd)), (l, i, j)
        bp = [b.copy() for b in bs]
        bm = [b.copy() for b in bs]
        bp[l][1] += eps
        bm[l][1] -= eps
        fd = (loss(Ws, bp) - loss(Ws, bm)) / (2 * eps)
        assert abs(fd - dbs[l][1]) < 1e-6 * max(1.0, abs(fd)), l
    # outputs past n_out carry no gradient
    assert np.all(dWs[2][n_out:] == 0) and np.all(dbs[2][n_out:] == 0)
