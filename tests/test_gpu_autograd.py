"""torch.autograd.Function over GPU rollouts: gradients match central finite differences, and forward
checkpointing with recomputation returns the same gradients as storing every step."""
import numpy as np
import pytest

from diffphd_b200 import scenes

pytestmark = pytest.mark.gpu


def _setup(ck):
    import torch
    from diffphd_b200.autograd import DiffSim
    sc = scenes.cantilever(cells=(4, 2, 2), dx=0.02, steps=6, heterogeneous=True)
    opts = dict(sc.options)
    opts.update(aa_window=0, rel_tol=1e-12, abs_tol=1e-14, max_pd_iter=5000)
    sim = DiffSim(sc, opts)
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev)
    return sc, sim, T


def _loss(sim, sc, T, q0, v0, params, f, r, ck):
    from diffphd_b200.autograd import Rollout
    qT, vT = Rollout.apply(sim, q0, v0, params, f, sc.steps, ck)
    return (qT * r).sum()


def test_autograd_matches_fd_and_checkpointing_is_exact():
    import torch
    sc, sim, T = _setup(2)
    r = T(np.random.default_rng(3).standard_normal(sc.dofs))
    grads = []
    for ck in (1, 2, 4):
        q0 = T(sc.q0).requires_grad_(True)
        v0 = T(sc.v0).requires_grad_(True)
        params = sim.default_params().to("cuda").requires_grad_(True)
        f = T(sc.f_ext).requires_grad_(True)
        L = _loss(sim, sc, T, q0, v0, params, f, r, ck)
        L.backward()
        grads.append((v0.grad.cpu().numpy(), params.grad.cpu().numpy(), f.grad.cpu().numpy()))
    for g in grads[1:]:
        for a, b in zip(g, grads[0]):
            assert np.array_equal(a, b)
    gv, gp, gf = grads[0]
    rng = np.random.default_rng(5)
    dv = rng.standard_normal(sc.dofs)
    dv[sc.dirichlet_dofs] = 0
    eps = 1e-5
    with torch.no_grad():
        p0 = sim.default_params().to("cuda")
        Lp = _loss(sim, sc, T, T(sc.q0), T(sc.v0 + eps * dv), p0, T(sc.f_ext), r, 3).item()
        Lm = _loss(sim, sc, T, T(sc.q0), T(sc.v0 - eps * dv), p0, T(sc.f_ext), r, 3).item()
        fd = (Lp - Lm) / (2 * eps)
        assert abs(gv @ dv - fd) <= 1e-4 * abs(fd)
        dp = rng.standard_normal(p0.numel()) * p0.cpu().numpy() * 1e-3
        Lp = _loss(sim, sc, T, T(sc.q0), T(sc.v0), p0 + T(dp), T(sc.f_ext), r, 3).item()
        Lm = _loss(sim, sc, T, T(sc.q0), T(sc.v0), p0 - T(dp), T(sc.f_ext), r, 3).item()
        fd = (Lp - Lm) / 2
        assert abs(gp @ dp - fd) <= 1e-3 * abs(fd)
        df = rng.standard_normal(sc.dofs)
        df[sc.dirichlet_dofs] = 0
        epsf = 1e-3
        Lp = _loss(sim, sc, T, T(sc.q0), T(sc.v0), p0, T(sc.f_ext + epsf * df), r, 3).item()
        Lm = _loss(sim, sc, T, T(sc.q0), T(sc.v0), p0, T(sc.f_ext - epsf * df), r, 3).item()
        fd = (Lp - Lm) / (2 * epsf)
        assert abs(gf @ df - fd) <= 1e-4 * abs(fd)


def test_checkpointed_contact_rollout_is_exact():
    """Through planar contact: recomputing segments from checkpoints (q, v and the contact multipliers) repeats
    the forward bit for bit, so every checkpoint interval gives the same gradients; the adjoint of each step
    finds its contact frame on the tape."""
    import torch
    from diffphd_b200.autograd import DiffSim, Rollout
    sc = scenes.contact_drop(cells=(3, 3, 3), dx=0.02, steps=8, height=0.0015, friction_mu=0.5)
    sc.q0 = sc.q0 + np.random.default_rng(11).normal(0.0, 2e-5, sc.q0.shape)
    opts = dict(sc.options)
    opts.update(aa_window=5, rel_tol=1e-10, abs_tol=1e-13, max_pd_iter=5000, friction_mu=0.5, alg_phd_bwd_solver=1)
    sim = DiffSim(sc, opts)
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev)
    r = T(np.random.default_rng(4).standard_normal(sc.dofs))
    grads = []
    for ck in (1, 3, 8):
        v0 = T(sc.v0).requires_grad_(True)
        params = sim.default_params().to("cuda").requires_grad_(True)
        qT, vT = Rollout.apply(sim, T(sc.q0), v0, params, T(sc.f_ext), sc.steps, ck)
        (qT * r).sum().backward()
        assert sim.deformable(params.detach().cpu().numpy()).contact_adjoint_stats()[0] == 1
        grads.append((v0.grad.cpu().numpy(), params.grad.cpu().numpy()))
    assert np.abs(grads[0][1]).max() > 0
    for g in grads[1:]:
        for a, b in zip(g, grads[0]):
            assert np.array_equal(a, b)


def test_checkpointed_rollout_with_learned_start_recomputes_exactly():
    """With a warm-start network attached, every checkpoint also holds the learned start's previous-step state, so
    recomputed segments repeat the forward pass bit for bit: gradients are identical for every checkpoint
    interval."""
    import torch
    from diffphd_b200.autograd import DiffSim
    from diffphd_b200.warmstart import WarmStartMLP
    sc = scenes.cantilever(cells=(4, 2, 2), dx=0.02, steps=7, heterogeneous=True)
    opts = dict(sc.options)
    opts.update(rel_tol=1e-8, abs_tol=1e-12, max_pd_iter=2000)
    dev = torch.device("cuda")
    sim = DiffSim(sc, opts, warm_start_network=WarmStartMLP(dev, seed=4))
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev)
    r = T(np.random.default_rng(8).standard_normal(sc.dofs))
    grads = []
    for ck in (1, 3, 7):
        q0 = T(sc.q0).requires_grad_(True)
        v0 = T(sc.v0).requires_grad_(True)
        params = sim.default_params().to("cuda").requires_grad_(True)
        L = _loss(sim, sc, T, q0, v0, params, T(sc.f_ext), r, ck)
        L.backward()
        grads.append((float(L.detach()), v0.grad.cpu().numpy(), params.grad.cpu().numpy()))
    for g in grads[1:]:
        assert g[0] == grads[0][0]
        assert np.array_equal(g[1], grads[0][1]) and np.array_equal(g[2], grads[0][2])
