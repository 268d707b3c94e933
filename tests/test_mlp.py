"""CPU checks of the surrogate's FP64 numpy restatement (the checker of the GPU MLP kernels)."""
import numpy as np
import torch

import mlp_numpy as M


def _random_case(n=64, seed=0):
    rng = np.random.default_rng(seed)
    p = rng.normal(0.0, 0.3, size=M.NPARAM)
    norm = np.concatenate([rng.normal(0, 1, 7), rng.uniform(0.5, 2.0, 7), [0.3, 1.7]])
    feats = rng.normal(0, 1, size=(n, 7))
    target = rng.normal(0, 1, size=n)
    return p, norm, feats, target


def test_loss_grad_matches_finite_differences():
    p, norm, feats, target = _random_case()
    _, g = M.loss_grad(p, norm, feats, target)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(np.arange(lo, hi), size=min(6, hi - lo), replace=False)
                          for lo, hi in M.GROUPS.values()])
    h = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += h
        lp, _ = M.loss_grad(q, norm, feats, target)
        q[i] -= 2 * h
        lm, _ = M.loss_grad(q, norm, feats, target)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(g[i]), (i, fd, g[i])


def test_bf16_round_matches_torch():
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.normal(0, 3, 10000), [1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, -2.5, 0.0]])
    x = x.astype(np.float32)
    ref = torch.tensor(x).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16_round(x), ref)


def test_infer_matches_unrounded_forward_closely():
    p, norm, feats, _ = _random_case(n=256, seed=3)
    y = M.infer_bf16(p, norm, feats)
    W1, b1, W2, b2, W3, b3 = M.unpack(p)
    x, _ = M.standardise(feats, None, norm)
    y64 = norm[14] + norm[15] * (M.gelu(M.gelu(x @ W1.T + b1) @ W2.T + b2) @ W3 + b3)
    assert np.max(np.abs(y - y64)) < 0.05 * (np.std(y64) + 1e-9)
