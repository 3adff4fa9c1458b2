"""The proposal network's CPU oracle: its backward pass against finite differences,
its AdamW step against torch.optim.AdamW, and its bf16 rounding (no GPU)."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from scipy.sparse import csr_matrix

from oracle import proposal_oracle as po


def _problem(seed=5, C=12, V=20, deg=4):
    rng = np.random.default_rng(seed)
    H = np.zeros((C, V), np.uint8)
    for c in range(C):
        H[c, rng.choice(V, deg, replace=False)] = 1
    H[:, 0] = 0                       # an isolated variable
    H[3, :] = 0                       # an empty check
    H[3, 7] = 1                       # ... then a degree-1 check
    g = po.Graph.from_csr(csr_matrix(H))
    B = 3
    syn = rng.integers(0, 2, (B, C)).astype(np.uint8)
    post = rng.normal(0, 6, (B, V))
    post[0, 1] = np.inf
    llr = np.full(V, 5.8)
    err = rng.integers(0, 2, (B, V)).astype(np.uint8)
    y = ((post <= 0).astype(np.uint8) == err).astype(np.uint8)
    return g, syn, post, llr, y


def test_layout_size():
    assert po.N_PARAMS == sum(int(np.prod(s)) for _, s in po.LAYOUT) == 4805


def test_backward_matches_finite_differences():
    g, syn, post, llr, y = _problem()
    theta = po.init_params(1).astype(np.float64)
    rng = np.random.default_rng(2)
    theta += rng.normal(0, 0.05, theta.shape)          # away from the symmetric start
    L, grad = po.backward(theta, g, syn, post, llr, y, w_neg=3.0, rounding=False)
    idx = np.concatenate([np.arange(o, o + min(12, int(np.prod(s)))) for o, s in po.offsets().values()])
    eps = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += eps
        tm[i] -= eps
        lp = po.loss_and_dr(po.forward(tp, g, syn, post, llr, rounding=False), y.astype(float), 3.0)[0]
        lm = po.loss_and_dr(po.forward(tm, g, syn, post, llr, rounding=False), y.astype(float), 3.0)[0]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, grad[i])


def test_adamw_matches_torch():
    rng = np.random.default_rng(0)
    theta = rng.normal(size=50)
    tp = torch.nn.Parameter(torch.tensor(theta))
    opt = torch.optim.AdamW([tp], lr=3e-3, betas=(0.9, 0.999), eps=1e-8, weight_decay=0.01)
    m = np.zeros_like(theta)
    v = np.zeros_like(theta)
    for step in range(1, 6):
        gnp = rng.normal(size=50)
        tp.grad = torch.tensor(gnp)
        opt.step()
        theta, m, v = po.adamw(theta, m, v, gnp, step, 3e-3)
    np.testing.assert_allclose(theta, tp.detach().numpy(), rtol=1e-12, atol=1e-12)


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(1).normal(0, 100, 10000)
    x[:3] = [1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -(1.0 + 2 ** -8)]  # ties to even
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).double().numpy()
    np.testing.assert_array_equal(po.bf16(x), ref)


def test_features_edge_cases():
    g, syn, post, llr, y = _problem()
    z, t, x = po.features(g, syn, post, llr)
    assert np.isfinite(z).all() and np.isfinite(x).all()
    assert z[0, 1, 0] == pytest.approx(1.0) and z[0, 1, 1] == 0.0      # +inf posterior clipped
    assert (x[:, :, 5] == 1).all()
    assert set(np.unique(t)) <= {0, 1, 2, 3}
    r = po.forward(po.init_params(0), g, syn, post, llr)
    assert r.shape == (3, g.V) and np.isfinite(r).all()
