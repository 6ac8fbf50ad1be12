"""The FP32 passes on a BF16 copy of the factor (option bf16_factor): every S / S^T pass of mixed precision is in
refinement form (x + S^T S (b - A x) with an FP64 residual) or a CG preconditioner, so a coarser factor changes the
iteration path, not the fixed point.  At tight gates the rollouts and adjoints match FP64."""
import numpy as np
import pytest

from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu

METHOD = "pd_eigen_alg_phd"


def _T(a, dev):
    import torch
    return torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev).contiguous()


def _rollout(d, sc, steps, opts, dev):
    import torch
    qs, vs = [_T(sc.q0, dev)], [_T(sc.v0, dev)]
    f = _T(sc.f_ext, dev)
    d.reset_frame_stats()
    for _ in range(steps):
        qn, vn = torch.empty_like(qs[0]), torch.empty_like(qs[0])
        d.forward_device(METHOD, qs[-1], vs[-1], f, sc.dt, opts, qn, vn)
        qs.append(qn)
        vs.append(vn)
    return qs, vs


def _sweep(d, sc, qs, opts, dev):
    import torch
    gq, gv = _T(sc.extra["loss_r"], dev), torch.zeros_like(qs[0])
    for i in reversed(range(len(qs) - 1)):
        dq, dv, df = torch.empty_like(gq), torch.empty_like(gq), torch.empty_like(gq)
        d.backward_device(METHOD, qs[i + 1], gq, gv, sc.dt, opts, dq, dv, df)
        gq, gv = dq, dv
    return gq.cpu().numpy(), gv.cpu().numpy()


def test_bf16_factor_rollout_and_adjoint_match_fp64_at_tight_gates():
    import torch
    dev = torch.device("cuda:0")
    sc = scenes.nh_tet_block(cells=(16, 8, 8), steps=8)
    tight = dict(sc.options, rel_tol=1e-10, abs_tol=1e-14, max_pd_iter=20000, alg_phd_bwd_solver=1)
    d64, d16 = core.from_scene(sc), core.from_scene(sc)
    q64, _ = _rollout(d64, sc, sc.steps, tight, dev)
    assert np.all(d64.frame_stats()[1] == 1)
    o16 = dict(tight, fp32_bulk=1, bf16_factor=1)
    q16, _ = _rollout(d16, sc, sc.steps, o16, dev)
    assert np.all(d16.frame_stats()[1] == 1)
    a, b = q16[-1].cpu().numpy(), q64[-1].cpu().numpy()
    disp = np.abs(b - sc.q0).max()
    err = np.abs(a - b).max() / disp
    print(f"bf16 factor rollout vs FP64: {err:.2e} of the displacement")
    assert err <= 1e-6
    # adjoints around each rollout's own states (equal to 1e-6): the BF16 factor only preconditions the
    # FP64-residual CG
    g64 = _sweep(d64, sc, q64, tight, dev)
    g16 = _sweep(d16, sc, q16, o16, dev)
    for x, y in zip(g16, g64):
        e = np.abs(x - y).max() / np.abs(y).max()
        print(f"bf16 factor adjoint vs FP64: {e:.2e}")
        assert e <= 1e-5


def test_bf16_factor_contact_rollout_has_the_fp64_contact_sets():
    sc = scenes.contact_drop(cells=(3, 3, 3), dx=0.02, steps=20, height=0.004, friction_mu=0.0)
    opts = dict(sc.options, friction_mu=0.0)
    d64, d16 = core.from_scene(sc), core.from_scene(sc)
    q, v = sc.q0.copy(), sc.v0.copy()
    touched = 0
    for _ in range(sc.steps):
        q6, v6, a6 = np.zeros(sc.dofs), np.zeros(sc.dofs), []
        q3, v3, a3 = np.zeros(sc.dofs), np.zeros(sc.dofs), []
        d64.PyForward(METHOD, q, v, [], sc.f_ext, sc.dt, opts, q6, v6, a6)
        d16.PyForward(METHOD, q, v, [], sc.f_ext, sc.dt, dict(opts, fp32_bulk=1, bf16_factor=1), q3, v3, a3)
        assert sorted(a3) == sorted(a6)
        touched += len(a6) > 0
        assert np.abs(q3 - q6).max() <= 1e-4 * np.abs(q6 - sc.q0).max()
        q, v = q6, v6
    assert touched > 0
