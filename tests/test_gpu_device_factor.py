"""Device construction of the sparse-inverse factor (separator chains built on the GPU from the Schur complement
of their descendants) against the host construction (the reference's LDL^T route, SparseLDLT.cpp:226-347): the
same A^-1 = S^T S to rounding, in FP64 and FP32, on hex and tet meshes, and the same contact rollouts."""
import numpy as np
import pytest

from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu


def _pair(sc, small_max):
    dh = core.from_scene(sc)
    dh.set_factor_build(1)
    dd = core.from_scene(sc)
    dd.set_factor_build(2, small_max)
    return dh, dd


@pytest.mark.parametrize("name,small_max", [("cantilever", 32), ("tet", 40), ("hex12", 64), ("hex12", 8)])
def test_device_factor_matches_host_factor(name, small_max):
    if name == "cantilever":
        sc = scenes.cantilever(steps=1)
    elif name == "tet":
        sc = scenes.nh_tet_block(cells=(12, 6, 6), steps=1)
    else:
        sc = scenes.contact_drop(cells=(12, 12, 12), steps=1)
    dh, dd = _pair(sc, small_max)
    rng = np.random.default_rng(3)
    for _ in range(2):
        b = rng.standard_normal(sc.dofs)
        xh = dh.debug_ainv(b, sc.dt)
        xd = dd.debug_ainv(b, sc.dt)
        assert dd.factor_built_on_device() and not dh.factor_built_on_device()
        assert dd.s_nnz() == dh.s_nnz()
        assert np.abs(xd - xh).max() <= 1e-12 * np.abs(xh).max()
        xh32 = dh.debug_ainv(b, sc.dt, fp32=True)
        xd32 = dd.debug_ainv(b, sc.dt, fp32=True)
        assert np.abs(xd32 - xh32).max() <= 2e-6 * np.abs(xh).max()


def test_device_factor_contact_rollout_matches_host():
    sc = scenes.hetero_contact(cells=(10, 10, 10), dx=0.01, steps=12, height=0.002)
    dh, dd = _pair(sc, 32)
    opts = dict(sc.options)
    # a tight gate: both factors then converge to the same fixed point, rounding apart
    opts.update(rel_tol=1e-11, abs_tol=1e-14, max_pd_iter=4000)
    qs = []
    for d in (dh, dd):
        q, v = sc.q0.copy(), sc.v0.copy()
        for _ in range(sc.steps):
            qn, vn = np.zeros(sc.dofs), np.zeros(sc.dofs)
            d.PyForward("pd_eigen_alg_phd", q, v, [], sc.f_ext, sc.dt, opts, qn, vn, [])
            q, v = qn, vn
        qs.append((q, d.frame_stats()[0], d.contact_lambda().cpu().numpy()))
    (qh, ith, lh), (qd, itd, ld) = qs
    assert np.count_nonzero(lh) > 0  # the block reached the ground
    assert np.array_equal(lh > 0, ld > 0)
    disp = np.abs(qh - sc.q0).max()
    assert np.abs(qd - qh).max() <= 1e-7 * disp
