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
