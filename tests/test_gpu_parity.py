"""GPU parity of the CUDA path against the CPU oracle, through the C ABI (run with -m gpu on a B200).

Tolerances: FP64 device path — A^-1 and local step 1e-12 relative, rollouts 1e-9 (plain PD, tight gate)
and 1e-6 (Anderson-accelerated, 1e-6 dual gate); adjoint 1e-8 relative to the oracle's adjoint; FP32 bulk
A^-1 5e-6 relative.
"""
import numpy as np
import pytest

import oracle
from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


SMALL = [
    lambda: scenes.cantilever(cells=(6, 2, 3), steps=1),
    lambda: scenes.cantilever(steps=1),
    lambda: scenes.nh_tet_block(cells=(8, 4, 4), dx=0.01, steps=1),
    lambda: scenes.nh_tet_block(steps=1),
]


@pytest.mark.parametrize("builder", SMALL)
def test_ainv_fp64_matches_oracle(builder):
    sc = builder()
    d = core.from_scene(sc)
    o = oracle.OracleDeformable.from_scene(sc)
    b = np.random.default_rng(1).standard_normal(sc.dofs)
    xr = o.ainv(b, sc.dt)
    xr[sc.dirichlet_dofs] = 0.0
    assert _rel(d.debug_ainv(b, sc.dt), xr) < 1e-12
    x32 = d.debug_ainv(b, sc.dt, fp32=True)
    assert _rel(x32, xr) < 5e-5


@pytest.mark.parametrize("builder", SMALL)
def test_local_step_matches_oracle(builder):
    sc = builder()
    d = core.from_scene(sc)
    o = oracle.OracleDeformable.from_scene(sc)
    rng = np.random.default_rng(2)
    q = sc.q0 + 0.02 * np.abs(sc.verts).max() * rng.standard_normal(sc.dofs) * 0.05
    q[sc.dirichlet_dofs] = sc.dirichlet_vals
    r = d.debug_local_step(q, sc.dt)
    rr = o.local_step(q)
    assert _rel(r, rr) < 1e-11


def _rollout_gpu(d, sc, steps, opts):
    q, v = sc.q0.copy(), sc.v0.copy()
    qs, vs = [q], [v]
    for _ in range(steps):
        qn, vn = np.zeros(sc.dofs), np.zeros(sc.dofs)
        d.PyForward("pd_eigen_alg_phd", q, v, [], sc.f_ext, sc.dt, opts, qn, vn, [])
        q, v = qn, vn
        qs.append(q)
        vs.append(v)
    return qs, vs


@pytest.mark.parametrize("aa", [0, 5])
def test_forward_rollout_cantilever(aa):
    sc = scenes.cantilever(steps=10)
    opts = dict(sc.options)
    if aa == 0:
        opts.update(aa_window=0, rel_tol=1e-10, abs_tol=1e-12, max_pd_iter=5000)
        tol = 1e-9
    else:
        opts.update(aa_window=5, rel_tol=1e-6, max_pd_iter=1000)
        tol = 1e-5
    d = core.from_scene(sc)
    o = oracle.OracleDeformable.from_scene(sc)
    qs, _ = _rollout_gpu(d, sc, 10, opts)
    q_ref, _, it_ref = oracle.rollout(o, sc, steps=10, options=opts)
    disp = np.abs(q_ref - sc.q0).max()
    assert np.abs(qs[-1] - q_ref).max() <= tol * max(disp, 1e-12)
    it_gpu, _ = d.frame_stats()
    assert len(it_gpu) == 10


def test_forward_rollout_nh_tets():
    sc = scenes.nh_tet_block(cells=(8, 4, 4), dx=0.01, steps=5)
    opts = dict(sc.options)
    opts.update(aa_window=0, rel_tol=1e-10, abs_tol=1e-12, max_pd_iter=5000)
    d = core.from_scene(sc)
    o = oracle.OracleDeformable.from_scene(sc)
    qs, _ = _rollout_gpu(d, sc, 5, opts)
    q_ref, _, _ = oracle.rollout(o, sc, steps=5, options=opts)
    disp = np.abs(q_ref - sc.q0).max()
    assert np.abs(qs[-1] - q_ref).max() <= 1e-8 * disp


@pytest.mark.parametrize("builder", [
    lambda: scenes.cantilever(cells=(4, 2, 2), dx=0.02, steps=3, heterogeneous=True),
    lambda: scenes.nh_tet_block(cells=(4, 2, 2), dx=0.01, steps=3),
])
def test_backward_matches_oracle(builder):
    sc = builder()
    opts = dict(sc.options)
    opts.update(aa_window=0, rel_tol=1e-12, abs_tol=1e-14, max_pd_iter=5000)
    o = oracle.OracleDeformable.from_scene(sc)
    q, v, _, qs, vs = oracle.rollout(o, sc, steps=sc.steps, options=opts, record=True)
    d = core.from_scene(sc)
    rng = np.random.default_rng(4)
    gq, gv = rng.standard_normal(sc.dofs), rng.standard_normal(sc.dofs) * 0.1
    i = sc.steps - 1
    ref = o.backward(qs[i], vs[i], sc.f_ext, sc.dt, qs[i + 1], gq, gv, opts)
    out = d.backward("pd_eigen_alg_phd", qs[i], vs[i], [], sc.f_ext, sc.dt, qs[i + 1], vs[i + 1], [], gq, gv, opts)
    for key in ("dl_dq", "dl_dv", "dl_df_ext"):
        assert _rel(out[key], ref[key]) < 1e-8, key
    assert _rel(out["dl_dstate_p"], ref["dl_dstate_p"]) < 1e-8
    assert _rel(out["dl_dmat_w"], ref["dl_dmat_w"]) < 1e-8
    assert _rel(out["dl_dparams"], np.concatenate(ref["dl_dparams"])) < 1e-7


def test_adjoint_matches_finite_differences_on_gpu():
    sc = scenes.cantilever(cells=(4, 2, 2), dx=0.02, steps=3, heterogeneous=True)
    opts = dict(sc.options)
    opts.update(aa_window=0, rel_tol=1e-12, abs_tol=1e-14, max_pd_iter=5000)
    r = np.random.default_rng(3).standard_normal(sc.dofs)

    def run(v0=None, params=None):
        s2 = sc
        d = core.HexDeformable()
        d.Initialize(sc.verts, sc.elems, sc.density, "none", 0, 0)
        for dof, val in zip(sc.dirichlet_dofs, sc.dirichlet_vals):
            d.SetDirichletBoundaryCondition(int(dof), float(val))
        ens = sc.energies if params is None else [(k, p, i) for (k, _, i), p in zip(sc.energies, params)]
        for k, p, i in ens:
            d.AddPdEnergy(k, p, i)
        d.AddStateForce("gravity", sc.gravity)
        q, v = sc.q0.copy(), (sc.v0 if v0 is None else v0).copy()
        qs, vs = [q], [v]
        for _ in range(s2.steps):
            qn, vn = np.zeros(sc.dofs), np.zeros(sc.dofs)
            d.PyForward("pd_eigen_alg_phd", q, v, [], sc.f_ext, sc.dt, opts, qn, vn, [])
            q, v = qn, vn
            qs.append(q)
            vs.append(v)
        return q @ r, d, qs, vs

    L, d, qs, vs = run()
    gq, gv = r.copy(), np.zeros(sc.dofs)
    gp = [np.zeros(np.size(p)) for _, p, _ in sc.energies]
    for i in reversed(range(sc.steps)):
        out = d.backward("pd_eigen_alg_phd", qs[i], vs[i], [], sc.f_ext, sc.dt, qs[i + 1], vs[i + 1], [], gq, gv,
                         opts)
        gq, gv = out["dl_dq"], out["dl_dv"]
        sizes = np.cumsum([np.size(p) for _, p, _ in sc.energies])[:-1]
        for a, b in zip(gp, np.split(out["dl_dparams"], sizes)):
            a += b
    dirn = np.random.default_rng(5).standard_normal(sc.dofs)
    dirn[sc.dirichlet_dofs] = 0
    eps = 1e-5
    fd = (run(v0=sc.v0 + eps * dirn)[0] - run(v0=sc.v0 - eps * dirn)[0]) / (2 * eps)
    assert abs(gv @ dirn - fd) <= 1e-4 * abs(fd)
    p0 = np.asarray(sc.energies[0][1], float)
    dp = np.random.default_rng(6).standard_normal(p0.size) * p0 * 1e-3
    ps = lambda s: [p0 + s * dp] + [np.asarray(p, float) for _, p, _ in sc.energies[1:]]
    fd = (run(params=ps(1))[0] - run(params=ps(-1))[0]) / 2
    assert abs(gp[0] @ dp - fd) <= 1e-3 * abs(fd)


def test_singular_element_reports_error():
    sc = scenes.cantilever(cells=(2, 1, 1), steps=1)
    d = core.from_scene(sc)
    q = sc.q0.copy().reshape(-1, 3)
    q[:, 0] = 0.0  # flatten the mesh: every F is singular
    with pytest.raises(RuntimeError, match="Singular F"):
        d.debug_local_step(q.ravel(), sc.dt)


def test_device_entry_points_match_host_entry_points():
    import torch
    sc = scenes.nh_tet_block(cells=(8, 4, 4), dx=0.01, steps=2)
    opts = dict(sc.options)
    d = core.from_scene(sc)
    qn_h, vn_h = np.zeros(sc.dofs), np.zeros(sc.dofs)
    d.PyForward("pd_eigen_alg_phd", sc.q0, sc.v0, [], sc.f_ext, sc.dt, opts, qn_h, vn_h, [])
    dev = torch.device("cuda")
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev).contiguous()
    qn, vn = torch.empty(sc.dofs, dtype=torch.float64, device=dev), torch.empty(sc.dofs, dtype=torch.float64,
                                                                                device=dev)
    s = torch.cuda.Stream()
    d.forward_device("pd_eigen_alg_phd", T(sc.q0), T(sc.v0), T(sc.f_ext), sc.dt, opts, qn, vn, stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(qn.cpu().numpy(), qn_h) and np.array_equal(vn.cpu().numpy(), vn_h)
    g = np.random.default_rng(0).standard_normal(sc.dofs)
    ref = d.backward("pd_eigen_alg_phd", sc.q0, sc.v0, [], sc.f_ext, sc.dt, qn_h, vn_h, [], g, 0 * g, opts)
    dq, dv, df = (torch.empty(sc.dofs, dtype=torch.float64, device=dev) for _ in range(3))
    dpar = torch.empty(d.NumOfPdParams(), dtype=torch.float64, device=dev)
    d.backward_device("pd_eigen_alg_phd", qn, T(g), T(0 * g), sc.dt, opts, dq, dv, df, dl_dparams=dpar,
                      stream=s.cuda_stream)
    s.synchronize()
    assert np.array_equal(dq.cpu().numpy(), ref["dl_dq"])
    assert np.array_equal(dpar.cpu().numpy(), ref["dl_dparams"])
    assert d.kernel_launches() > 0


@pytest.mark.parametrize("fp32", [0, 1])
def test_pcg_adjoint_matches_converged_oracle_adjoint(fp32):
    """The conjugate-gradient adjoint (FP64 residual against A, S^T S preconditioner in FP64 or FP32) reaches
    the converged adjoint of the oracle to 1e-7 in FP64.  In mixed precision the K_pd apply also runs in FP32
    (packed symmetric per-sample Jacobians), so the converged adjoint carries that operator's rounding: 5e-6
    (measured about 1e-6 on this block)."""
    sc = scenes.nh_tet_block(cells=(6, 3, 3), dx=0.01, steps=2)
    opts = dict(sc.options)
    opts.update(aa_window=0, rel_tol=1e-13, abs_tol=1e-16, max_pd_iter=20000)
    o = oracle.OracleDeformable.from_scene(sc)
    q, v, _, qs, vs = oracle.rollout(o, sc, steps=2, options=opts, record=True)
    rng = np.random.default_rng(8)
    gq, gv = rng.standard_normal(sc.dofs), rng.standard_normal(sc.dofs) * 0.1
    ref = o.backward(qs[1], vs[1], sc.f_ext, sc.dt, qs[2], gq, gv, opts)
    d = core.from_scene(sc)
    gopts = dict(opts, alg_phd_bwd_solver=1, fp32_bulk=fp32, rel_tol=1e-12, max_pd_iter=2000)
    out = d.backward("pd_eigen_alg_phd", qs[1], vs[1], [], sc.f_ext, sc.dt, qs[2], vs[2], [], gq, gv, gopts)
    assert out["iters"] < 2000
    tol, ptol = (5e-6, 1e-5) if fp32 else (1e-7, 1e-6)
    errs = {key: _rel(out[key], ref[key]) for key in ("dl_dq", "dl_dv", "dl_df_ext")}
    errs["dl_dparams"] = _rel(out["dl_dparams"], np.concatenate(ref["dl_dparams"]))
    print("relative errors vs the oracle:", errs)
    for key in ("dl_dq", "dl_dv", "dl_df_ext"):
        assert errs[key] < tol, (key, errs[key])
    assert errs["dl_dparams"] < ptol, errs["dl_dparams"]


def test_mixed_precision_forward_error_vs_fp64():
    """Precision of the mixed path in isolation: FP64 and mixed (FP32 projection delta, FP32 S^T S in
    refinement form with the FP64 residual against A) each run exactly 3000 plain PD iterations per step (gate
    disabled), which converges this block to its fixed point; the two fixed points differ by < 1e-5 of the
    displacement after 3 steps.  The FP64 run is also checked against the oracle at the same settings."""
    sc = scenes.nh_tet_block(cells=(8, 4, 4), dx=0.01, steps=3)
    opts = dict(sc.options)
    opts.update(aa_window=0, rel_tol=0.0, abs_tol=0.0, max_pd_iter=3000, verbose=-1)
    d64 = core.from_scene(sc)
    q64, _ = _rollout_gpu(d64, sc, 3, opts)
    d32 = core.from_scene(sc)
    q32, _ = _rollout_gpu(d32, sc, 3, dict(opts, fp32_bulk=1))
    o = oracle.OracleDeformable.from_scene(sc)
    q_ref, _, _ = oracle.rollout(o, sc, steps=3, options=dict(opts, verbose=0))
    disp = np.abs(q_ref - sc.q0).max()
    assert np.abs(q64[-1] - q_ref).max() <= 1e-9 * disp
    assert np.abs(q32[-1] - q64[-1]).max() <= 1e-5 * disp
