"""Learned warm start on the GPU: the fused BF16 tensor-core MLP kernels against the numpy oracle (forward,
loss gradient, AdamW), the feature / target kernels against numpy, the warm-started PD loop against the plain
one (same gate, same fixed point), and what a network trained on solver rollouts gains in PD iterations."""
import numpy as np
import pytest

from diffphd_b200 import scenes
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _dev():
    import torch
    return torch.device("cuda:0")


def _mlp(seed=0, scale=None):
    from diffphd_b200.warmstart import WarmStartMLP
    mlp = WarmStartMLP(_dev(), seed=seed)
    if scale is not None:
        rng = np.random.default_rng(seed)
        mlp.load_master(rng.standard_normal(M.N_PARAMS) * scale)
    return mlp


def _batch(n, seed=0):
    import torch
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 16))
    X[:, 15] = 0
    Xb = torch.as_tensor(X, dtype=torch.float32).to(torch.bfloat16).to(_dev())
    Y = rng.standard_normal((n, 4)) * 0.2
    return Xb, torch.as_tensor(Y, dtype=torch.float32, device=_dev()), M.bf16(X), Y


@pytest.mark.parametrize("n", [1, 127, 1000, 4096])
def test_mlp_forward_matches_oracle(n):
    mlp = _mlp(1, scale=0.15)
    Xb, _, X, _ = _batch(n, 2)
    out = mlp.forward(Xb).cpu().numpy().astype(np.float64)
    ref, _ = M.forward(mlp.master.cpu().numpy(), X, emulate=True)
    err = np.abs(out - ref).max() / max(np.abs(ref).max(), 1e-30)
    assert err < 2e-3, err


@pytest.mark.parametrize("n", [200, 3000])
def test_mlp_gradient_matches_oracle(n):
    mlp = _mlp(3, scale=0.1)
    Xb, Y, X, Yn = _batch(n, 4)
    loss, grad = mlp.gradient(Xb, Y)
    l_ref, g_ref = M.loss_and_grad(mlp.master.cpu().numpy(), X, Y.cpu().numpy(), emulate=True)
    g = grad.cpu().numpy().astype(np.float64)
    assert abs(float(loss) - l_ref) <= 1e-4 * abs(l_ref)
    assert np.all(g[~M.used_mask()] == 0)
    rel = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert rel < 5e-3, rel
    # against the exact FP64 network: the BF16 operands' cost, stated
    _, g64 = M.loss_and_grad(mlp.master.cpu().numpy(), X, Y.cpu().numpy(), emulate=False)
    assert np.linalg.norm(g - g64) / np.linalg.norm(g64) < 5e-2


def test_mlp_gradient_is_deterministic():
    mlp = _mlp(5, scale=0.1)
    Xb, Y, _, _ = _batch(5000, 6)
    _, g1 = mlp.gradient(Xb, Y)
    _, g2 = mlp.gradient(Xb, Y)
    assert np.array_equal(g1.cpu().numpy(), g2.cpu().numpy())


def test_adamw_step_matches_oracle():
    import torch
    mlp = _mlp(7, scale=0.1)
    Xb, Y, _, _ = _batch(700, 8)
    w0 = mlp.master.cpu().numpy().astype(np.float64)
    lr, wd = 3e-3, 0.01
    for step in range(1, 4):
        _, g = mlp.gradient(Xb, Y)
        m0, v0 = mlp.m.cpu().numpy().astype(np.float64), mlp.v.cpu().numpy().astype(np.float64)
        w_before = mlp.master.cpu().numpy().astype(np.float64)
        grad = torch.zeros_like(mlp.master)
        mlp.train_step(Xb, Y, lr, weight_decay=wd, grad=grad)
        assert np.array_equal(grad.cpu().numpy(), g.cpu().numpy())
        w_ref, m_ref, v_ref = M.adamw(w_before, g.cpu().numpy().astype(np.float64), m0, v0, step, lr,
                                      weight_decay=wd)
        np.testing.assert_allclose(mlp.master.cpu().numpy(), w_ref, rtol=2e-6, atol=1e-7)
        np.testing.assert_allclose(mlp.m.cpu().numpy(), m_ref, rtol=1e-5, atol=1e-6 * np.abs(m_ref).max())
    assert not np.array_equal(mlp.master.cpu().numpy(), w0)
    # the BF16 operand copies follow the masters
    out = mlp.forward(Xb).cpu().numpy()
    ref, _ = M.forward(mlp.master.cpu().numpy(), M.bf16(Xb.float().cpu().numpy()), emulate=True)
    assert np.abs(out - ref).max() < 2e-3 * np.abs(ref).max()


def test_training_fits_a_smooth_map():
    """Training through the fused kernels drives the loss of a smooth 16 -> 4 map down by an order of magnitude."""
    import torch
    from diffphd_b200.warmstart import fit
    rng = np.random.default_rng(9)
    N = 60000
    X = rng.uniform(-1, 1, (N, 16))
    Y = np.stack([np.sin(2 * X[:, 0]) * X[:, 1], X[:, 2] ** 2 - X[:, 3], np.tanh(X[:, 4] + X[:, 5] * X[:, 6]),
                  np.maximum(X[:, 15], 0) * X[:, 7]], axis=1) * 0.1
    Xb = torch.as_tensor(X, dtype=torch.float32).to(torch.bfloat16).to(_dev())
    Yt = torch.as_tensor(Y, dtype=torch.float32, device=_dev())
    mlp = _mlp(10)
    l0 = float(mlp.gradient(Xb, Yt)[0])
    fit(mlp, Xb, Yt, steps=400, batch=8192, lr=3e-3)
    l1 = float(mlp.gradient(Xb, Yt)[0])
    assert l1 < 0.1 * l0, (l0, l1)


def _scene(seed, steps=30):
    return scenes.nh_tet_block(cells=(12, 6, 6), dx=0.01, steps=steps, seed=seed)


def test_features_base_and_target_kernels():
    import torch
    from diffphd_b200 import core
    sc = _scene(0)
    d = core.from_scene(sc)
    dev = _dev()
    n3 = sc.dofs
    rng = np.random.default_rng(11)
    q = torch.as_tensor(sc.q0 + rng.standard_normal(n3) * 1e-3, device=dev)
    qp = torch.as_tensor(sc.q0 + rng.standard_normal(n3) * 1e-3, device=dev)
    v = torch.as_tensor(rng.standard_normal(n3) * 0.1, device=dev)
    f = torch.as_tensor(rng.standard_normal(n3) * 1e-3, device=dev)
    pb = torch.as_tensor(sc.q0 + rng.standard_normal(n3) * 1e-3, device=dev)
    qn, vn = torch.empty_like(q), torch.empty_like(q)
    d.forward_device("pd_eigen_alg_phd", q, v, f, sc.dt, sc.options, qn, vn)
    X = torch.empty(n3 // 3, 16, dtype=torch.bfloat16, device=dev)
    base = torch.empty_like(q)
    d.warmstart_features(sc.dt, q, qp, v, f, pb, X, base)
    nodes = n3 // 3
    # reference quantities
    vol = 0.01 ** 3 / 5.0
    mass = sc.density * vol
    dx = vol ** (1.0 / 3.0)
    h = sc.dt
    g = np.array([0, 0, -9.81])
    qq, qpp, vv, ff, pbb = (t.cpu().numpy() for t in (q, qp, v, f, pb))
    base_ref = qq + h * vv + h * h / mass * ff + h * h * np.tile(g, nodes)
    np.testing.assert_allclose(base.cpu().numpy(), base_ref, rtol=1e-14, atol=1e-15)
    Xn = X.float().cpu().numpy()
    exp = np.zeros((nodes, 16))
    exp[:, 0:3] = ((qq - sc.q0) / dx).reshape(-1, 3)
    exp[:, 3:6] = ((qq - qpp) / dx).reshape(-1, 3)
    exp[:, 6:9] = ((qq - pbb) / dx).reshape(-1, 3)
    exp[:, 9:12] = (h * h / mass * ff / dx).reshape(-1, 3)
    fixed = np.zeros(nodes, bool)
    fixed[np.asarray(sc.dirichlet_dofs) // 3] = True
    exp[:, 14] = fixed
    np.testing.assert_allclose(Xn[:, :12], M.bf16(exp[:, :12]), rtol=0, atol=1e-6)
    assert np.array_equal(Xn[:, 14], exp[:, 14])
    assert np.all(Xn[:, 12] == 0) and np.all(Xn[:, 15] == 0)
    assert np.all(Xn[:, 13] > 0.5) and np.all(Xn[:, 13] < 1.1)  # log10(stiffness)/7 for 1e5..1e7 Pa
    Y = torch.empty(nodes, 4, dtype=torch.float32, device=dev)
    d.warmstart_target(sc.dt, qn, base, Y)
    np.testing.assert_allclose(Y.cpu().numpy()[:, :3].ravel(),
                               ((qn.cpu().numpy() - base_ref) / dx).astype(np.float32), rtol=1e-6, atol=1e-7)
    assert np.all(Y.cpu().numpy()[:, 3] == 0)  # no contact set: the multiplier target is zero
    # q_init = base + dx * out, Dirichlet dofs at their values
    out = torch.as_tensor(rng.standard_normal((nodes, 8)) * 0.1, dtype=torch.float32, device=dev)
    qi = torch.empty_like(q)
    d.warmstart_apply(sc.dt, base, out, qi)
    exp_qi = base_ref + dx * out[:, :3].cpu().numpy().astype(np.float64).ravel()
    exp_qi[np.asarray(sc.dirichlet_dofs)] = np.asarray(sc.dirichlet_vals)
    np.testing.assert_allclose(qi.cpu().numpy(), exp_qi, rtol=1e-15, atol=1e-15)


def test_warm_started_loop_reaches_the_plain_fixed_point():
    """A start away from q (here the inertial prediction q_tilde, and a half-way point with noise) converges to
    the plain loop's fixed point at the gate."""
    import torch
    from diffphd_b200 import core
    sc = _scene(1)
    d = core.from_scene(sc)
    dev = _dev()
    opts = dict(sc.options)
    opts.update(rel_tol=1e-10, abs_tol=1e-13, max_pd_iter=5000)
    q = torch.as_tensor(sc.q0, device=dev)
    v = torch.zeros_like(q)
    f = torch.zeros_like(q)
    qa, va, qb, vb = (torch.empty_like(q) for _ in range(4))
    d.forward_device("pd_eigen_alg_phd", q, v, f, sc.dt, opts, qa, va)
    disp = float((qa - q).abs().max())
    rng = np.random.default_rng(12)
    X = torch.empty(sc.n, 16, dtype=torch.bfloat16, device=dev)
    base = torch.empty_like(q)
    d.warmstart_features(sc.dt, q, q, v, f, None, X, base)
    half = q + 0.5 * (qa - q) * (1 + torch.as_tensor(rng.standard_normal(sc.dofs) * 0.1, device=dev))
    for qi in (base, half):
        d.forward_device_init("pd_eigen_alg_phd", q, v, f, sc.dt, opts, qi, qb, vb)
        # both loops stop at the gate; their distance is the gate's accuracy (rel_tol / (1 - contraction))
        assert float((qa - qb).abs().max()) <= 1e-4 * disp
    it, cv = d.frame_stats()
    assert np.all(cv == 1), (it, cv)


def _bench_scene(seed):
    return scenes.nh_tet_block(seed=seed)


def test_learned_warm_start_reduces_pd_iterations():
    """A network trained on plain-solver rollouts of 6 held-out material fields of the 32x16x16 tet block starts
    the PD loop closer to its fixed point on 2 other fields: fewer iterations at the same dual gate.  The
    attached-network path (PyForward / forward_device) gives the same trajectory as the explicit stepper."""
    import torch
    from diffphd_b200 import core
    from diffphd_b200.warmstart import WarmStartMLP, WarmStartStepper, evaluate, fit, generate_dataset
    dev = _dev()
    X, Y = generate_dataset(_bench_scene, seeds=range(1, 7), steps=50, device=dev)
    mlp = WarmStartMLP(dev, seed=0)
    fit(mlp, X, Y, steps=1000, batch=65536, lr=2e-3)
    del X, Y
    res = evaluate(_bench_scene, seeds=[100, 101], steps=40, mlp=mlp, device=dev, modes=("plain", "learned"))
    plain, learned = np.mean(res["plain"]["iters"]), np.mean(res["learned"]["iters"])
    print("PD iterations per step, plain vs learned start:", res["plain"]["iters"], res["learned"]["iters"])
    assert learned < 0.9 * plain, (plain, learned)
    # attached network == explicit stepper, bit for bit
    sc = _bench_scene(100)
    d = core.from_scene(sc)
    q0 = torch.as_tensor(sc.q0, device=dev)
    v0 = torch.zeros_like(q0)
    f = torch.zeros_like(q0)
    finals = []
    for attached in (False, True):
        d.reset_warm_start()
        d.set_warm_start_network(mlp if attached else None)
        st = None if attached else WarmStartStepper(d, mlp, "pd_eigen_alg_phd", sc.dt, sc.options)
        q, v = q0.clone(), v0.clone()
        for _ in range(5):
            qn, vn = torch.empty_like(q), torch.empty_like(q)
            if attached:
                d.forward_device("pd_eigen_alg_phd", q, v, f, sc.dt, sc.options, qn, vn)
            else:
                st.step(q, v, f, qn, vn)
            q, v = qn, vn
        finals.append(q.cpu().numpy())
    d.set_warm_start_network(None)
    assert np.array_equal(finals[0], finals[1])
