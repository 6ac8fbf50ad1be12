"""GPU parity of the planar Signorini–Coulomb contact path against the oracle (run with -m gpu on a B200).

A 3x3x3-cell block falls 4 mm onto z = 0 (every node a candidate).  With plain PD at a tight gate the
rollouts agree to 1e-7 of the displacement and the per-step active contact sets are identical; with the
reference defaults (Anderson window 5, 1e-6 gate) they agree to 1e-4 of the displacement.
"""
import numpy as np
import pytest

import oracle
from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu


def _roll_gpu(d, sc, steps, opts):
    q, v = sc.q0.copy(), sc.v0.copy()
    acts = []
    for _ in range(steps):
        qn, vn, act = np.zeros(sc.dofs), np.zeros(sc.dofs), []
        d.PyForward("pd_eigen_alg_phd", q, v, [], sc.f_ext, sc.dt, opts, qn, vn, act)
        q, v = qn, vn
        acts.append(sorted(act))
    return q, v, acts


def _roll_oracle(o, sc, steps, opts):
    q, v = sc.q0.copy(), sc.v0.copy()
    acts = []
    o.reset_warm_start()
    for _ in range(steps):
        q, v, act = o.forward(q, v, sc.f_ext, sc.dt, opts)
        acts.append(sorted(act.tolist()))
    return q, v, acts


@pytest.mark.parametrize("mu", [0.0, 0.5])
def test_contact_rollout_matches_oracle_tight(mu):
    sc = scenes.contact_drop(cells=(3, 3, 3), dx=0.02, steps=30, height=0.004, friction_mu=mu)
    opts = dict(sc.options)
    opts.update(aa_window=0, rel_tol=1e-11, abs_tol=1e-14, max_pd_iter=8000, friction_mu=mu)
    o = oracle.OracleDeformable.from_scene(sc)
    q_ref, _, acts_ref = _roll_oracle(o, sc, sc.steps, opts)
    d = core.from_scene(sc)
    q, _, acts = _roll_gpu(d, sc, sc.steps, opts)
    assert any(len(a) for a in acts_ref), "the block never touched the plane"
    assert acts == acts_ref
    disp = np.abs(q_ref - sc.q0).max()
    assert np.abs(q - q_ref).max() <= 1e-7 * disp
    z = q.reshape(-1, 3)[:, 2]
    assert z.min() > -1e-3


def test_contact_rollout_matches_oracle_reference_defaults():
    sc = scenes.contact_drop(cells=(3, 3, 3), dx=0.02, steps=30, height=0.004, friction_mu=0.5)
    opts = dict(sc.options)
    opts.update(max_pd_iter=1000)
    o = oracle.OracleDeformable.from_scene(sc)
    q_ref, _, _ = _roll_oracle(o, sc, sc.steps, opts)
    d = core.from_scene(sc)
    q, _, _ = _roll_gpu(d, sc, sc.steps, opts)
    disp = np.abs(q_ref - sc.q0).max()
    assert np.abs(q - q_ref).max() <= 1e-4 * disp


def test_contact_mixed_precision_vs_fp64():
    """Contact in mixed precision (FP32 projections and S/S^T passes in refinement form, FP64 NCP solve and
    residual), with a fixed number of PD iterations per step (gate disabled, so both precisions reach their
    fixed points).  Frictionless, the 20-step rollout stays within 2e-6 of the FP64 one with the same active
    sets (measured 2e-7 per step).  With friction the Coulomb stick/slip law amplifies FP32 rounding, so each
    mixed step is compared from the same FP64 input state: within 2e-4 of the displacement from rest
    (measured 9e-5 at worst over 14 steps)."""
    sc = scenes.contact_drop(cells=(3, 3, 3), dx=0.02, steps=20, height=0.004, friction_mu=0.0)
    opts = dict(sc.options)
    opts.update(aa_window=0, rel_tol=0.0, abs_tol=0.0, max_pd_iter=2000, friction_mu=0.0, verbose=-1)
    q64, _, acts64 = _roll_gpu(core.from_scene(sc), sc, sc.steps, opts)
    q32, _, acts32 = _roll_gpu(core.from_scene(sc), sc, sc.steps, dict(opts, fp32_bulk=1))
    assert any(len(a) for a in acts64), "the block never touched the plane"
    assert acts32 == acts64
    assert np.abs(q32 - q64).max() <= 2e-6 * np.abs(q64 - sc.q0).max()

    sc = scenes.contact_drop(cells=(3, 3, 3), dx=0.02, steps=14, height=0.004, friction_mu=0.5)
    opts.update(friction_mu=0.5)
    d64, d32 = core.from_scene(sc), core.from_scene(sc)
    q, v = sc.q0.copy(), sc.v0.copy()
    touched, worst = 0, 0.0
    for _ in range(sc.steps):
        q6, v6, a6 = np.zeros(sc.dofs), np.zeros(sc.dofs), []
        q3, v3, a3 = np.zeros(sc.dofs), np.zeros(sc.dofs), []
        d64.PyForward("pd_eigen_alg_phd", q, v, [], sc.f_ext, sc.dt, opts, q6, v6, a6)
        d32.PyForward("pd_eigen_alg_phd", q, v, [], sc.f_ext, sc.dt, dict(opts, fp32_bulk=1), q3, v3, a3)
        assert sorted(a3) == sorted(a6)
        touched += len(a6) > 0
        worst = max(worst, np.abs(q3 - q6).max() / np.abs(q6 - sc.q0).max())
        q, v = q6, v6
    print("worst per-step mixed vs FP64 difference / displacement from rest:", worst)
    assert touched > 0
    assert worst <= 2e-4


def test_cached_factor_ncp_solve_matches_fresh_factorisation():
    """The NCP's dense solve by CG preconditioned with a cached factor (ncp_solver 1, the default) against a fresh
    Cholesky at every PD iteration (ncp_solver 0, the reference's scheme): the same active sets and the same
    rollout, on a block whose whole bottom face rests on the ground.  At this 1e-10 gate some frames reach the
    3000-iteration cap (a cycle of active-set flips at the 1e-10 level), so the two rollouts agree only to the
    amplified CG rounding: 1.5e-6 and 2.2e-5 of the displacement with two builds of the cached solve, measured on
    a B200."""
    sc = scenes.hetero_contact(cells=(12, 12, 12), dx=0.01, steps=16, height=5e-4)
    out = []
    for solver in (0, 1):
        d = core.from_scene(sc)
        opts = dict(sc.options, ncp_solver=solver, rel_tol=1e-10, abs_tol=1e-14, max_pd_iter=3000)
        q, v, acts = _roll_gpu(d, sc, sc.steps, opts)
        out.append((q, acts, d.ncp_solve_stats(detail=True)))
    (q0, a0, s0), (q1, a1, s1) = out
    assert a0 == a1 and len(a1[-1]) == 13 * 13
    assert s0 == (0, 0, 0, 0)                # ncp_solver 0 never touches the cached factor
    assert s1[1] > 0 and s1[0] > 3 * s1[1]   # mostly solved by the cached factor
    assert s1[2] > 0
    disp = np.abs(q0 - sc.q0).max()
    assert np.abs(q1 - q0).max() <= 1e-4 * disp


def test_contact_frame_recomputes_bit_for_bit():
    """Every frame starts without a cached NCP factor: the same frame computed again from the same state and
    multipliers gives the same bits (what the checkpointed backward relies on), in mixed precision too."""
    import torch
    sc = scenes.hetero_contact(cells=(12, 12, 12), dx=0.01, steps=6, height=5e-4)
    d = core.from_scene(sc)
    dev = torch.device("cuda:0")
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev).contiguous()
    q, v, f = T(sc.q0), T(sc.v0), T(sc.f_ext)
    for fp32 in (0, 1):
        opts = dict(sc.options, fp32_bulk=fp32)
        for _ in range(5):
            qn, vn = torch.empty_like(q), torch.empty_like(q)
            d.forward_device("pd_eigen_alg_phd", q, v, f, sc.dt, opts, qn, vn)
            q, v = qn, vn
        lam = d.contact_lambda().clone()
        outs = []
        for _ in range(2):
            d.set_contact_lambda(lam)
            qn, vn = torch.empty_like(q), torch.empty_like(q)
            d.forward_device("pd_eigen_alg_phd", q, v, f, sc.dt, opts, qn, vn)
            outs.append((qn, vn, d.contact_lambda().clone()))
        assert (lam > 0).any()
        for a, b in zip(*outs):
            assert torch.equal(a, b)
