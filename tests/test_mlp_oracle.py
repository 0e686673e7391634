"""The prefilter's CPU oracle itself (no GPU)."""
import numpy as np
import torch

import mlp_oracle as mo


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(10000).astype(np.float32) * 10,
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.0078125, 65504.0, 1e-30], dtype=np.float32)])
    want = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(mo.bf16(x), want)


def test_oracle_gradient_matches_float64_without_rounding():
    # with BF16 rounding removed, the closed-form gradient must match a float64 autograd gradient
    rng = np.random.default_rng(1)
    k = 9
    theta = mo.init_like(seed=1, k=k).astype(np.float64)
    kmers = rng.integers(0, 2**63, size=64, dtype=np.int64).astype(np.uint64) * np.uint64(2)
    labels = (rng.random(64) < 0.5).astype(np.float64)
    t = torch.tensor(theta, requires_grad=True)
    W1 = t[0:32768].reshape(256, 128)
    b1 = t[32768:33024]
    W2 = t[33024:98560].reshape(256, 256)
    b2 = t[98560:98816]
    w3 = t[98816:99072]
    b3 = t[99072]
    X = torch.tensor(mo.onehot(kmers, k), dtype=torch.float64)
    z = torch.relu(torch.relu(X @ W1.T + b1) @ W2.T + b2) @ w3 + b3
    y = torch.tensor(labels)
    loss = torch.mean(torch.nn.functional.softplus(z) - y * z)
    loss.backward()
    saved = mo.bf16
    mo.bf16 = lambda a: np.asarray(a, dtype=np.float64)
    try:
        l2, g = mo.loss_and_grad(theta, kmers, labels, k)
    finally:
        mo.bf16 = saved
    assert abs(l2 - loss.item()) < 1e-5
    assert np.allclose(g, t.grad.numpy(), rtol=1e-4, atol=1e-6)
