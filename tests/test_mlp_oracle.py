"""The numpy MLP oracle pinned against independent references: central finite differences of its FP64
loss, torch's own AdamW, and its BF16 rounding against torch's BF16 conversion (CPU only)."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def _params(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal(M.N_PARAMS) * scale
    return p


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.standard_normal(20000) * 10.0 ** rng.integers(-6, 6, 20000),
                        [0.0, -0.0, 1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 65504.0, 1e-30]])
    ref = torch.as_tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16(x), ref)


def test_fp64_gradient_matches_central_differences():
    rng = np.random.default_rng(2)
    n = 37
    X = rng.standard_normal((n, 16))
    X[:, 15] = 0.0
    Y = rng.standard_normal((n, 4))
    p = _params(3)
    _, g = M.loss_and_grad(p, X, Y, emulate=False)
    used = M.used_mask()
    assert np.all(g[~used] == 0)
    idx = np.concatenate([rng.choice(np.arange(M.OFF_W1, M.OFF_W2)[used[M.OFF_W1:M.OFF_W2]], 12),
                          rng.choice(np.arange(M.OFF_W2, M.OFF_W3), 12),
                          rng.choice(np.arange(M.OFF_W3, M.OFF_B1)[used[M.OFF_W3:M.OFF_B1]], 12),
                          rng.choice(np.arange(M.OFF_B1, M.OFF_B3), 12), [M.OFF_B3, M.OFF_B3 + 2]])
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (M.loss_and_grad(pp, X, Y, emulate=False)[0] - M.loss_and_grad(pm, X, Y, emulate=False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_fp64_forward_matches_torch_network():
    import torch
    rng = np.random.default_rng(4)
    X = rng.standard_normal((50, 16))
    p = _params(5)
    W1, W2, W3, b1, b2, b3 = M.unpack(p)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64)
    gelu = torch.nn.GELU(approximate="none")
    out = gelu(gelu(t(X) @ t(W1) + t(b1)) @ t(W2) + t(b2)) @ t(W3) + t(b3)
    ref, _ = M.forward(p, X, emulate=False)
    np.testing.assert_allclose(ref, out.numpy(), rtol=1e-12, atol=1e-12)


def test_adamw_matches_torch():
    import torch
    rng = np.random.default_rng(6)
    p = _params(7)
    used = M.used_mask()
    decay = np.zeros(M.N_PARAMS, bool)
    decay[:M.OFF_B1] = True
    lr, wd = 1e-2, 0.05
    tw = torch.nn.Parameter(torch.as_tensor(p[used & decay]))
    tb = torch.nn.Parameter(torch.as_tensor(p[used & ~decay]))
    opt = torch.optim.AdamW([{"params": [tw], "weight_decay": wd}, {"params": [tb], "weight_decay": 0.0}],
                            lr=lr, betas=(0.9, 0.999), eps=1e-8)
    w, m, v = p.copy(), np.zeros_like(p), np.zeros_like(p)
    for step in range(1, 6):
        g = rng.standard_normal(M.N_PARAMS)
        g[~used] = 0
        w, m, v = M.adamw(w, g, m, v, step, lr, weight_decay=wd)
        tw.grad = torch.as_tensor(g[used & decay])
        tb.grad = torch.as_tensor(g[used & ~decay])
        opt.step()
    np.testing.assert_allclose(w[used & decay], tw.detach().numpy(), rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(w[used & ~decay], tb.detach().numpy(), rtol=1e-12, atol=1e-14)
    assert np.array_equal(w[~used], p[~used])


def test_emulated_gradient_is_close_to_fp64():
    """BF16 operands cost about 1% of the gradient; the emulation is what the GPU is compared with."""
    rng = np.random.default_rng(8)
    X = rng.standard_normal((300, 16))
    X[:, 15] = 0
    Y = rng.standard_normal((300, 4)) * 0.1
    p = _params(9, 0.1)
    _, g64 = M.loss_and_grad(p, X, Y, emulate=False)
    _, g16 = M.loss_and_grad(p, X, Y, emulate=True)
    assert np.linalg.norm(g16 - g64) <= 0.05 * np.linalg.norm(g64)
