"""Parity at the configured sizes (not shrunken meshes), through the C ABI, against the FP64 oracle.

  * the 32x16x16 Neo-Hookean tet block (40,960 tets) for 20 steps with the bench's options -- FP32 bulk, learned
    PD warm start, adjoint warm start, Anderson window 5, the 1e-6 dual gate: the FP64 path against the oracle at
    a 1e-10 gate (relative position error <= 1e-6), the bench's path no further from the converged trajectory
    than the oracle at the 1e-6 gate, and its reverse sweep against the oracle's (gradient error <= 1e-4);
  * the 16x4x4 cantilever (425 nodes) for 100 steps: gradients w.r.t. q0, v0 and the per-element Young's moduli
    (through the Lame chain of the per-element energy parameters) against central differences (eps chosen
    above the loss's convergence noise, see the test);
  * the 24^3 contact drop (rotated block, Coulomb mu 0.5, every node a candidate) for 24 steps in FP64: the same
    contact set as the oracle at every step (the oracle on an exactly prefiltered candidate set) and positions
    within the gate's accuracy;
  * the reference's own backward (mean stiffness inside K_pd, deformable_projective_dynamics_backward.cpp:37-44,
    option bwd_mean_stiffness) against the oracle in the same mode.
"""
import numpy as np
import pytest

from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu

METHOD = "pd_eigen_alg_phd"


def _T(a, dev):
    import torch
    return torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev).contiguous()


def _gpu_rollout(d, sc, steps, opts, dev):
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


def test_tet_block_bench_options_match_the_fp64_oracle(oracle_lib):
    """The 32x16x16 tet block for 20 steps with the bench's options.

    The reference's stop rule (step <= rel_tol |q|, forward_gpu.cpp:1381-1397) measures the last PD step, and PD
    converges slowly on this stiff block, so at rel_tol 1e-6 every frame stops about 1e-3 (relative position) short
    of its fixed point: the oracle itself after 5 steps is 1.0e-3 from its 1e-10 solution, 8.4e-6 at 1e-8 (measured
    here on the CPU).  Two iteration paths that pass the same 1e-6 gate -- even the FP64 GPU path and the oracle
    from the same start, whose A^-1 roundings differ -- therefore differ by that much (6e-4 measured on a B200
    after 20 steps).  So parity is checked where it is defined:
      * the FP64 path against the oracle at a 1e-10 gate (both at their fixed points) for the first steps:
        positions within 1e-6;
      * the bench's path (FP32 bulk, learned start, adjoint warm start) at the 1e-6 gate against the converged
        trajectory (the FP64 path at the 1e-10 gate): no further from it than the oracle at the 1e-6 gate;
      * the bench's adjoint (PCG, mixed precision, warm-started) over the last 3 steps of the reverse sweep,
        around its own forward states, against the oracle's FP64 adjoint around the same states at a 1e-9 gate:
        relative gradient error <= 1e-4.  (The reference's adjoint fixed point with its default 500-iteration
        cap is not converged on this block: 210% from its 1e-10 solution after 3 steps, 3.5e-4 with 5000
        iterations, measured here on the CPU -- hence the converged oracle as the yardstick.)"""
    import torch
    from diffphd_b200.warmstart import WarmStartMLP, fit, generate_dataset
    dev = torch.device("cuda:0")
    steps, tight_steps, bwd_steps = 20, 2, 3
    sc = scenes.nh_tet_block(steps=steps)  # 32 x 16 x 16 cells, 9,537 nodes
    base = dict(sc.options, thread_ct=16)
    mixed = dict(base, fp32_bulk=1, alg_phd_bwd_solver=1, alg_phd_bwd_warm_start=3)
    tight = dict(base, rel_tol=1e-10, abs_tol=1e-14, max_pd_iter=20000)
    tight_bwd = dict(base, rel_tol=1e-9, abs_tol=1e-14, max_pd_iter=20000)
    # a briefly trained warm-start network (held-out material seeds), attached as in the bench
    X, Y = generate_dataset(lambda s: scenes.nh_tet_block(seed=s), [1, 2], 8, dev, options=base)
    mlp = WarmStartMLP(dev, seed=0)
    fit(mlp, X, Y, steps=300, batch=32768, lr=2e-3)
    d64 = core.from_scene(sc)
    qstar, _ = _gpu_rollout(d64, sc, steps, tight, dev)
    assert np.all(d64.frame_stats()[1] == 1)
    d = core.from_scene(sc)
    d.set_warm_start_network(mlp)
    qs, vs = _gpu_rollout(d, sc, steps, mixed, dev)
    assert np.all(d.frame_stats()[1] == 1)
    r = sc.extra["loss_r"]
    gq, gv = _T(r, dev), torch.zeros_like(qs[0])
    gpar = np.zeros(d.NumOfPdParams())
    dpar = torch.empty(d.NumOfPdParams(), dtype=torch.float64, device=dev)
    for i in reversed(range(steps - bwd_steps, steps)):
        dq, dv, df = torch.empty_like(gq), torch.empty_like(gq), torch.empty_like(gq)
        d.backward_device(METHOD, qs[i + 1], gq, gv, sc.dt, mixed, dq, dv, df, dl_dparams=dpar)
        gpar += dpar.cpu().numpy()
        gq, gv = dq, dv
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    o = oracle_lib.OracleDeformable.from_scene(sc)
    q, v = sc.q0.copy(), sc.v0.copy()
    for k in range(tight_steps):
        q, v, _ = o.forward(q, v, sc.f_ext, sc.dt, tight)
    err_fp64 = rel(qstar[tight_steps].cpu().numpy(), q)
    q, v = sc.q0.copy(), sc.v0.copy()
    for _ in range(steps):
        q, v, _ = o.forward(q, v, sc.f_ext, sc.dt, base)
    q_star = qstar[-1].cpu().numpy()
    err_ref_gate = rel(q, q_star)
    err_bench = rel(qs[-1].cpu().numpy(), q_star)
    print(f"tet block: FP64 path vs oracle at the 1e-10 gate after {tight_steps} steps {err_fp64:.2e}; after 20 steps, "
          f"from the converged trajectory: oracle at the 1e-6 gate {err_ref_gate:.2e}, bench path {err_bench:.2e}")
    assert err_fp64 <= 1e-6
    assert err_bench <= max(err_ref_gate, 1e-6)
    # the adjoint: the oracle's FP64 reverse sweep around the bench path's forward states, over the last steps,
    # converged (a 1e-9 gate)
    qn = [x.cpu().numpy() for x in qs]
    vn = [x.cpu().numpy() for x in vs]
    g, g_v = r.copy(), np.zeros(sc.dofs)
    opar = np.zeros(d.NumOfPdParams())
    for i in reversed(range(steps - bwd_steps, steps)):
        out = o.backward(qn[i], vn[i], sc.f_ext, sc.dt, qn[i + 1], g, g_v, tight_bwd)
        opar += np.concatenate(out["dl_dparams"])
        g, g_v = out["dl_dq"], out["dl_dv"]
    for name, a, b in (("dl_dq", gq.cpu().numpy(), g), ("dl_dv", gv.cpu().numpy(), g_v), ("dl_dparams", gpar, opar)):
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        print(f"  {name}: relative error {err:.2e}")
        assert err <= 1e-4, (name, err)


def _cantilever_loss(sim, sc, q0, v0, params, steps):
    import torch
    from diffphd_b200.autograd import Rollout
    dev = q0.device
    qT, _ = Rollout.apply(sim, q0, v0, params, _T(sc.f_ext, dev), steps, 10)
    return (qT * _T(sc.extra["loss_r"], dev)).sum()


def test_cantilever_100_steps_gradients_match_central_differences():
    """Gradients of r . q_100 through 100 steps of the heterogeneous cantilever w.r.t. v0, q0 and the per-element
    Young's moduli, against central differences of the same GPU rollout.

    The forward runs to a 1e-12 gate: the loss then moves by 2.5e-9 between the 1e-11 and 1e-12 gates (the
    oracle, measured here on the CPU; 3,000-15,000 PD iterations per frame), so its noise is ~1e-10 and a
    central difference resolves 1e-4 only where 2 eps |dL| is above ~1e-6.  Implicit Euler damps a random
    velocity field's high modes within the 100 steps (dL/dv0 along one is ~3e-5), so the directions are the
    cantilever's first bending shape for v0 and q0 and a random relative field for E, with eps 1e-2 (a 1 cm/s
    tip velocity, a 10 um tip offset: both in the linear regime of a sag of centimetres) and 1e-3 for E."""
    import torch
    from diffphd_b200.autograd import DiffSim
    dev = torch.device("cuda:0")
    sc = scenes.cantilever(steps=100, heterogeneous=True)  # 16 x 4 x 4 hex cells, per-element E
    opts = dict(sc.options, rel_tol=1e-12, abs_tol=1e-14, max_pd_iter=30000, alg_phd_bwd_solver=1)
    sim = DiffSim(sc, opts)
    q0 = _T(sc.q0, dev).requires_grad_(True)
    v0 = _T(sc.v0, dev).requires_grad_(True)
    p0 = sim.default_params().to(dev).requires_grad_(True)
    L = _cantilever_loss(sim, sc, q0, v0, p0, sc.steps)
    L.backward()
    gq0, gv0, gp = q0.grad.cpu().numpy(), v0.grad.cpu().numpy(), p0.grad.cpu().numpy()
    sizes = sim.sizes
    dE, _ = scenes.chain_material_grad(sc, np.split(gp, np.cumsum(sizes)[:-1]))
    free = np.ones(sc.dofs, bool)
    free[sc.dirichlet_dofs] = False
    x = sc.verts[:, 0] - sc.verts[:, 0].min()
    bend = np.zeros((sc.n, 3))
    bend[:, 2] = x / x.max()  # first bending shape: vertical, growing from the clamped face
    bend = bend.ravel() * free
    rng = np.random.default_rng(3)
    with torch.no_grad():
        def loss(q0n=sc.q0, v0n=sc.v0, E=sc.youngs):
            params = np.concatenate([np.atleast_1d(p) for _, p, _ in scenes.energy_params_from_material(sc, E)])
            return float(_cantilever_loss(sim, sc, _T(q0n, dev), _T(v0n, dev), _T(params, dev), sc.steps))
        for name, grad, direction, eps, fn in (
                ("v0", gv0, bend, 1e-2, lambda t, dv: loss(v0n=sc.v0 + t * dv)),
                ("q0", gq0, bend * 1e-3, 1e-2, lambda t, dq: loss(q0n=sc.q0 + t * dq)),
                ("E", dE, rng.standard_normal(sc.m) * sc.youngs, 1e-3, lambda t, de: loss(E=sc.youngs + t * de))):
            fd = (fn(eps, direction) - fn(-eps, direction)) / (2 * eps)
            an = float(grad @ direction)
            print(f"cantilever 100 steps, d/d{name}: adjoint {an:.9e}  FD {fd:.9e}")
            assert abs(an - fd) <= 1e-4 * abs(fd), (name, an, fd)


def test_contact_drop_24_cubed_has_the_oracles_contact_sets(oracle_lib):
    """The 24^3 drop with every node a candidate runs on the GPU; the oracle, whose Delassus block is dense over its
    candidates (a 15,625^2 block of A^-1 columns per step), runs the same rollout on the 628 nodes that start
    within 6 cells of the lowest one (the GPU puts nodes up to 3.34 cells above it in contact) -- asserted: every
    node the full GPU rollout ever puts in contact is among them.  The GPU on that candidate set and the oracle
    then have the same contact set at every step and positions within the gate's accuracy, up to the first frame
    whose PD loop does not converge: from frame 17 on, the coupled PD / NCP iteration with Coulomb friction
    cycles in some frames (5,000 iterations do not settle it, measured on a B200), and two runs whose roundings
    differ -- even the GPU on the full and on the prefiltered candidate list -- then part ways."""
    import copy
    sc = scenes.contact_drop(height=0.002, steps=24)  # 24^3 hex block, seeded rotation, Coulomb mu 0.5
    opts = dict(sc.options, thread_ct=16, max_pd_iter=2000)
    z0 = sc.q0.reshape(-1, 3)[:, 2]
    sub = np.nonzero(z0 <= z0.min() + 6.0 * 0.01)[0]
    sc_sub = copy.copy(sc)
    sc_sub.plane = (sc.plane[0], sub)

    def gpu_rollout(scene):
        d = core.from_scene(scene)
        q, v = scene.q0.copy(), scene.v0.copy()
        qs, acts = [], []
        for _ in range(scene.steps):
            qn, vn = np.zeros(scene.dofs), np.zeros(scene.dofs)
            d.PyForward(METHOD, q, v, [], scene.f_ext, scene.dt, opts, qn, vn, [])
            q, v = qn, vn
            lam = d.contact_lambda().cpu().numpy()
            qs.append(q)
            acts.append(set(np.asarray(scene.plane[1])[lam > 0].tolist()))
        return qs, acts, d.frame_stats()[1]

    q_all, a_all, _ = gpu_rollout(sc)
    assert sum(bool(a) for a in a_all) >= 20           # at least 20 steps with contact
    assert set().union(*a_all) <= set(sub.tolist())     # the prefilter loses no contact
    q_sub, a_sub, conv = gpu_rollout(sc_sub)
    o = oracle_lib.OracleDeformable.from_scene(sc_sub)
    qo, vo = sc.q0.copy(), sc.v0.copy()
    compared = 0
    for t in range(sc.steps):
        qo, vo, act_o = o.forward(qo, vo, sc.f_ext, sc.dt, opts)
        if not (conv[t] and o.last_converged):
            break
        assert a_sub[t] == set(act_o.tolist()), (t, len(a_sub[t]), len(act_o))
        assert np.abs(q_sub[t] - qo).max() <= 1e-4 * np.abs(qo - sc.q0).max()
        compared += bool(a_sub[t])
    print(f"24^3 drop: identical contact sets on {compared} contact steps before the first unconverged frame")
    assert compared >= 10


def test_reference_mean_stiffness_backward_matches_the_oracle(oracle_lib):
    sc = scenes.cantilever(cells=(8, 2, 2), dx=0.02, steps=1, heterogeneous=True)
    opts = dict(sc.options, aa_window=0, rel_tol=1e-12, abs_tol=1e-14, max_pd_iter=5000, bwd_mean_stiffness=1)
    d = core.from_scene(sc)
    qn, vn = np.zeros(sc.dofs), np.zeros(sc.dofs)
    d.PyForward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, opts, qn, vn, [])
    g = np.random.default_rng(4).standard_normal(sc.dofs)
    o = oracle_lib.OracleDeformable.from_scene(sc)
    qo, _, _ = o.forward(sc.q0, sc.v0, sc.f_ext, sc.dt, opts)
    for solver in (0, 1):
        out = d.backward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, qn, vn, [], g, 0 * g,
                         dict(opts, alg_phd_bwd_solver=solver))
        ref = o.backward(sc.q0, sc.v0, sc.f_ext, sc.dt, qo, g, 0 * g, opts)
        for k in ("dl_dq", "dl_dv", "dl_df_ext"):
            assert np.abs(out[k] - ref[k]).max() <= 1e-7 * np.abs(ref[k]).max(), (solver, k)
        a, b = np.asarray(out["dl_dparams"]).ravel(), np.concatenate(ref["dl_dparams"])
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max(), solver
        # the mean-stiffness adjoint is not the exact one: it differs from the default (per-element) adjoint
        exact = d.backward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, qn, vn, [], g, 0 * g,
                           dict(opts, bwd_mean_stiffness=0, alg_phd_bwd_solver=solver))
        assert np.abs(exact["dl_dv"] - out["dl_dv"]).max() > 1e-6 * np.abs(out["dl_dv"]).max()
