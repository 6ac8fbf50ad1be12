"""Adjoint through planar contact on the GPU against the oracle (run with -m gpu on a B200).

The oracle restates the reference's backward literally: the forward tape, its pop or a replayed forward step,
the backbone adjoint by the Anderson fixed point, and the contact-aware material adjoint
z_q = mu - W_T G_T^-1 J mu with one fixed-point solve per contact basis vector.  The GPU solves the same
constrained system by one projected conjugate-gradient run.  At a tight gate (inner solves converged) both give
the same dl_dq, dl_dv, dl_df_ext and material gradients.
"""
import numpy as np
import pytest

import oracle
from diffphd_b200 import core, scenes

pytestmark = pytest.mark.gpu
M = "pd_eigen_alg_phd"


def _setup(mu, steps=9):
    sc = scenes.contact_drop(cells=(3, 3, 3), dx=0.02, steps=steps, height=0.0015, friction_mu=mu)
    # A slightly strained start: a rigid block has repeated singular values (sigma = 1, 1, 1) in every element,
    # where the reference's SVD-derivative guard makes the volume projection's differential discontinuous and
    # the adjoint ill-conditioned; the perturbation keeps the comparison away from that degenerate state.
    sc.q0 = sc.q0 + np.random.default_rng(11).normal(0.0, 2e-5, sc.q0.shape)
    fwd = dict(sc.options)
    fwd.update(aa_window=0, rel_tol=1e-11, abs_tol=1e-14, max_pd_iter=8000, friction_mu=mu)
    bwd = dict(fwd)
    bwd.update(aa_window=5, alg_phd_bwd_wt_max_iter=20000, max_pd_iter=20000, alg_phd_bwd_solver=1)
    return sc, fwd, bwd


def _forward_both(sc, fwd, steps):
    o = oracle.OracleDeformable.from_scene(sc)
    o.reset_warm_start()
    d = core.from_scene(sc)
    qo, vo = [sc.q0.copy()], [sc.v0.copy()]
    qg, vg = [sc.q0.copy()], [sc.v0.copy()]
    acts = []
    for _ in range(steps):
        q, v, act = o.forward(qo[-1], vo[-1], sc.f_ext, sc.dt, fwd)
        qo.append(q)
        vo.append(v)
        qn, vn, a = np.zeros(sc.dofs), np.zeros(sc.dofs), []
        d.PyForward(M, qg[-1], vg[-1], [], sc.f_ext, sc.dt, fwd, qn, vn, a)
        qg.append(qn)
        vg.append(vn)
        acts.append(len(act))
    return o, d, qo, vo, qg, vg, acts


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("mu", [0.0, 0.5])
def test_contact_adjoint_matches_oracle(mu):
    sc, fwd, bwd = _setup(mu)
    steps = sc.steps
    o, d, qo, vo, qg, vg, acts = _forward_both(sc, fwd, steps)
    assert sum(acts) > 0, "no contact during the rollout"
    r = np.random.default_rng(5).standard_normal(sc.dofs)
    go, gvo = r.copy(), np.zeros(sc.dofs)
    constrained = 0
    worst = {}
    for i in reversed(range(steps)):
        # both sides get the same upstream gradients (the oracle's), each its own trajectory (tape match)
        ref = o.backward(qo[i], vo[i], sc.f_ext, sc.dt, qo[i + 1], go, gvo, bwd)
        out = d.backward(M, qg[i], vg[i], [], sc.f_ext, sc.dt, qg[i + 1], vg[i + 1], [], go, gvo, bwd)
        source, cons, _ = d.contact_adjoint_stats()
        assert source == 1, "the backward did not find its forward frame on the tape"
        constrained += cons
        errs = {k: _rel(out[k], ref[k]) for k in ("dl_dq", "dl_dv", "dl_df_ext")}
        errs["dl_dparams"] = _rel(out["dl_dparams"], np.concatenate(ref["dl_dparams"]))
        for k, e in errs.items():
            worst[k] = max(worst.get(k, 0.0), e)
        go, gvo = ref["dl_dq"], ref["dl_dv"]
    print("worst relative error per output over the sweep:", worst)
    assert constrained > 0, "no contact constraint entered the material adjoint"
    for k, e in worst.items():
        assert e < 1e-6, (k, e)


def test_contact_adjoint_skip_option_and_replay():
    sc, fwd, bwd = _setup(0.5, steps=8)
    o, d, qo, vo, qg, vg, acts = _forward_both(sc, fwd, sc.steps)
    assert acts[-1] > 0
    r = np.random.default_rng(6).standard_normal(sc.dofs)
    z = np.zeros(sc.dofs)
    i = sc.steps - 1
    first = d.backward(M, qg[i], vg[i], [], sc.f_ext, sc.dt, qg[i + 1], vg[i + 1], [], r, z, bwd)
    assert d.contact_adjoint_stats()[0] == 1
    ref_first = o.backward(qo[i], vo[i], sc.f_ext, sc.dt, qo[i + 1], r, z, bwd)
    # the frame is gone from both tapes: a second call replays the forward step from (q, v, f_ext)
    again = d.backward(M, qg[i], vg[i], [], sc.f_ext, sc.dt, qg[i + 1], vg[i + 1], [], r, z, bwd)
    assert d.contact_adjoint_stats()[0] == 2
    ref_again = o.backward(qo[i], vo[i], sc.f_ext, sc.dt, qo[i + 1], r, z, bwd)
    assert _rel(again["dl_dparams"], np.concatenate(ref_again["dl_dparams"])) < 1e-6
    assert _rel(again["dl_dparams"], first["dl_dparams"]) < 1e-5
    assert _rel(first["dl_dparams"], np.concatenate(ref_first["dl_dparams"])) < 1e-6
    # skip_contact_woodbury: the material gradients use the plain adjoint mu, on both sides
    skip = dict(bwd)
    skip["skip_contact_woodbury"] = 1
    s_gpu = d.backward(M, qg[i], vg[i], [], sc.f_ext, sc.dt, qg[i + 1], vg[i + 1], [], r, z, skip)
    assert d.contact_adjoint_stats()[0] == 0
    s_ref = o.backward(qo[i], vo[i], sc.f_ext, sc.dt, qo[i + 1], r, z, skip)
    assert _rel(s_gpu["dl_dparams"], np.concatenate(s_ref["dl_dparams"])) < 1e-6
    assert _rel(s_gpu["dl_dq"], first["dl_dq"]) < 1e-8  # routing never uses the correction
    # skip_material_grad: zero material gradients
    nomat = dict(bwd)
    nomat["skip_material_grad"] = 1
    n_gpu = d.backward(M, qg[i], vg[i], [], sc.f_ext, sc.dt, qg[i + 1], vg[i + 1], [], r, z, nomat)
    assert np.all(n_gpu["dl_dparams"] == 0)
