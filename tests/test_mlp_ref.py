"""The CPU checker of the learned guess (oracle/mlp_ref.py): its backward
pass against central finite differences of its own forward pass (without
rounding, so the loss is smooth), and BF16 rounding against known values."""
import numpy as np

from oracle import mlp_ref


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.0, 0.0], dtype=np.float32)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1.0); 1.005859375
    # rounds up; 1 + 2^-7 is exact
    want = np.array([1.0, 1.0, 1.0078125, 1.0078125, -3.0, 0.0], dtype=np.float32)
    assert np.array_equal(mlp_ref.bf16r(x), want)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    nf, n = 8, 16
    _, P = mlp_ref.offsets(nf)
    params = rng.normal(scale=0.3, size=P)
    feats = rng.normal(size=(n, nf))
    tgt = rng.normal(size=(n, 2))
    loss, g = mlp_ref.loss_and_grad(params, feats, tgt, rounding=False)
    idx = rng.choice(P, 60, replace=False)
    for i in idx:
        h = 1e-6
        pp, pm = params.copy(), params.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = mlp_ref.loss_and_grad(pp, feats, tgt, rounding=False)
        lm, _ = mlp_ref.loss_and_grad(pm, feats, tgt, rounding=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
