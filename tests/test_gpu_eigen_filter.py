"""The state-adaptive eigen filter of the adjoint's local Hessians on the GPU against the oracle (-m gpu).

Each sample's 9x9 PD Hessian H = (sum w) I - J is kept when diagonally dominant and otherwise rebuilt from its
eigen-decomposition with the eigenvalues clamped at 0 (bwd_eigen_filter = 1) or replaced by their absolute
values (2), the rule of ProjectedNewtonMatrix (deformable_newton_forward.cpp:394-434).  A compressed
Neo-Hookean block has indefinite samples, so the filter changes the adjoint.
"""
import numpy as np
import pytest

import oracle
from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu
M = "pd_eigen_alg_phd"


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("filt", [1, 2])
def test_eigen_filtered_adjoint_matches_oracle(filt):
    sc = scenes.nh_tet_block(cells=(6, 3, 3), dx=0.01, steps=4, seed=2)
    # squeeze the block along x (every node moves towards the clamped face) to create compressed samples
    q0 = sc.q0.reshape(-1, 3).copy()
    q0[:, 0] *= 0.8
    sc.q0 = q0.ravel()
    opts = dict(sc.options)
    opts.update(aa_window=0, rel_tol=1e-12, abs_tol=1e-15, max_pd_iter=20000, alg_phd_bwd_solver=0)
    o = oracle.OracleDeformable.from_scene(sc)
    d = core.from_scene(sc)
    q, v = sc.q0.copy(), sc.v0.copy()
    qn, vn = np.zeros(sc.dofs), np.zeros(sc.dofs)
    d.PyForward(M, q, v, [], sc.f_ext, sc.dt, opts, qn, vn, [])
    qo, vo, _ = o.forward(q, v, sc.f_ext, sc.dt, opts)
    assert np.abs(qn - qo).max() <= 1e-8 * np.abs(qo - q).max()
    g = np.random.default_rng(3).standard_normal(sc.dofs)
    z = np.zeros(sc.dofs)
    results = {}
    for f in (0, filt):
        b = dict(opts)
        b["bwd_eigen_filter"] = f
        out = d.backward(M, q, v, [], sc.f_ext, sc.dt, qn, vn, [], g, z, b)
        ref = o.backward(q, v, sc.f_ext, sc.dt, qn, g, z, b)
        nf_gpu, nf_ref = d.last_filtered_samples(), o.last_filtered
        if f:
            assert nf_ref > 0 and abs(nf_gpu - nf_ref) <= max(2, nf_ref // 50), (nf_gpu, nf_ref)
        for key in ("dl_dq", "dl_dv"):
            assert _rel(out[key], ref[key]) < 1e-7, (f, key, _rel(out[key], ref[key]))
        assert _rel(out["dl_dparams"], np.concatenate(ref["dl_dparams"])) < 1e-6
        results[f] = out["dl_dq"]
    assert _rel(results[filt], results[0]) > 1e-6, "the filter did not change the adjoint"
