"""Failure paths of the GPU step, made on the host (no fault, trap or hang of the GPU): a non-finite input, a PD
loop capped before it converges, the conjugate-gradient adjoint's fallback to the reference fixed point, and a
tensor-core completion wait of the warm-start kernel that runs out.  After each one the handle keeps working.

Reference behaviour followed: CheckError -> RuntimeError (cpp/core/src/common/common.cpp:87-94); a PD loop that
reaches max_pd_iter is a warning with the frame marked unconverged
(cpp/core/src/fem/deformable_projective_dynamics_forward_gpu.cpp:1405-1408)."""
import numpy as np
import pytest

from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu

METHOD = "pd_eigen_alg_phd"


def _small():
    sc = scenes.cantilever(cells=(6, 2, 2), dx=0.02, steps=1, heterogeneous=True)
    return sc, core.from_scene(sc)


def test_non_finite_input_raises_and_the_handle_recovers():
    sc, d = _small()
    qn, vn = np.zeros(sc.dofs), np.zeros(sc.dofs)
    d.PyForward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, sc.options, qn, vn, [])
    q_ok = qn.copy()
    q_bad = sc.q0.copy()
    q_bad[3 * 7 + 1] = np.nan  # a free node's y
    with pytest.raises(RuntimeError, match="non-finite"):
        d.PyForward(METHOD, q_bad, sc.v0, [], sc.f_ext, sc.dt, sc.options, qn, vn, [])
    d.PyForward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, sc.options, qn, vn, [])
    assert np.array_equal(qn, q_ok)


def test_capped_pd_loop_reports_an_unconverged_frame(capfd):
    sc, d = _small()
    opts = dict(sc.options, max_pd_iter=1)
    qn, vn = np.zeros(sc.dofs), np.zeros(sc.dofs)
    d.PyForward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, opts, qn, vn, [])
    it, cv = d.frame_stats()
    assert list(it) == [1] and list(cv) == [0]
    assert "did not converge" in capfd.readouterr().err
    assert np.all(np.isfinite(qn))
    d.PyForward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, sc.options, qn, vn, [])
    assert d.frame_stats()[1][-1] == 1


def test_cg_fallback_to_the_fixed_point_gives_the_fixed_point_adjoint():
    sc, d = _small()
    opts = dict(sc.options, aa_window=0, rel_tol=1e-12, abs_tol=1e-14, max_pd_iter=5000)
    qn, vn = np.zeros(sc.dofs), np.zeros(sc.dofs)
    d.PyForward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, opts, qn, vn, [])
    g = np.random.default_rng(2).standard_normal(sc.dofs)
    ref = d.backward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, qn, vn, [], g, 0 * g, dict(opts, alg_phd_bwd_solver=0))
    before = d.backward_fallbacks()
    out = d.backward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, qn, vn, [], g, 0 * g,
                     dict(opts, alg_phd_bwd_solver=1, debug_force_bwd_fallback=1))
    assert d.backward_fallbacks() == before + 1
    for k in ("dl_dq", "dl_dv", "dl_df_ext"):
        assert np.abs(out[k] - ref[k]).max() <= 1e-12 * np.abs(ref[k]).max()


def test_tensor_core_wait_that_runs_out_is_an_error_not_a_hang():
    import torch
    from diffphd_b200.warmstart import WarmStartMLP
    L = core.load_library()
    dev = torch.device("cuda")
    mlp = WarmStartMLP(dev, seed=1)
    rng = np.random.default_rng(0)
    X = torch.as_tensor(rng.standard_normal((4096, 16)), dtype=torch.float32).to(torch.bfloat16).to(dev)
    ref = mlp.forward(X, tcgen05=True).clone()
    mlp.check_tensor_core_waits()
    try:
        assert L.dphd_debug_set_mma_wait_polls(0) == 0  # no poll: the first completion wait gives up
        mlp.forward(X, tcgen05=True)
        torch.cuda.synchronize()
        with pytest.raises(RuntimeError, match="timed out"):
            mlp.check_tensor_core_waits()
    finally:
        assert L.dphd_debug_set_mma_wait_polls(-1) == 0  # the default bound again
    out = mlp.forward(X, tcgen05=True)
    mlp.check_tensor_core_waits()
    assert torch.equal(out, ref)
    # the same flag stops a forward step that uses the attached network
    sc, d = _small()
    d.set_warm_start_network(mlp)
    try:
        assert L.dphd_debug_set_mma_wait_polls(0) == 0
        qn, vn = np.zeros(sc.dofs), np.zeros(sc.dofs)
        with pytest.raises(RuntimeError, match="timed out"):
            d.PyForward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, sc.options, qn, vn, [])
    finally:
        assert L.dphd_debug_set_mma_wait_polls(-1) == 0
    d.PyForward(METHOD, sc.q0, sc.v0, [], sc.f_ext, sc.dt, sc.options, qn, vn, [])
    assert np.all(np.isfinite(qn))
