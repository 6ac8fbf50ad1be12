"""CPU checks that pin the oracle (the CPU restatement used as the checker) before it is trusted.

* mesh layer: bit-exact against fixtures written by the reference's own mesher (tests/golden/)
* 3x3 SVD / polar: against LAPACK (numpy)
* projections: defining optimality conditions; differentials against central differences
* A^-1: against a dense solve of the assembled A
* adjoint: against central finite differences of the oracle forward
"""
from pathlib import Path

import numpy as np
import pytest

from diffphd_b200 import scenes
from diffphd_b200.mesh import generate_hex_mesh, hex_to_tet5, read_bin, write_bin

GOLD = Path(__file__).resolve().parent / "golden"


def test_hex_mesh_matches_reference_writer():
    v, e = read_bin(GOLD / "ref_hex_16x4x4.bin")
    v2, e2, _ = generate_hex_mesh(np.ones((16, 4, 4)), 0.01)
    assert np.array_equal(v, v2) and np.array_equal(e, e2)
    vox = np.ones((3, 3, 2))
    vox[1, 1, :] = 0
    vox[2, 0, 1] = 0
    v, e = read_bin(GOLD / "ref_hex_holes.bin")
    v2, e2, _ = generate_hex_mesh(vox, 0.5, [0.1, -0.2, 0.3])
    assert np.array_equal(v, v2) and np.array_equal(e, e2)


def test_bin_roundtrip_matches_reference_tet_writer(tmp_path):
    v, e = read_bin(GOLD / "ref_tet_2.bin")
    write_bin(tmp_path / "t.bin", v, e)
    assert (tmp_path / "t.bin").read_bytes() == (GOLD / "ref_tet_2.bin").read_bytes()


def test_tet5_split_conforming():
    v, h, ijk = generate_hex_mesh(np.ones((3, 2, 2)), 1.0)
    t = hex_to_tet5(v, h, ijk)
    assert t.shape == (60, 4)
    x = v[t]
    vol = np.einsum("ij,ij->i", np.cross(x[:, 1] - x[:, 0], x[:, 2] - x[:, 0]), x[:, 3] - x[:, 0]) / 6
    assert np.all(vol > 0)
    assert abs(vol.sum() - 12.0) < 1e-12
    # conforming: every interior triangle is shared by exactly two tets
    faces = {}
    for tet in t:
        for f in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)):
            key = tuple(sorted(tet[list(f)]))
            faces[key] = faces.get(key, 0) + 1
    assert max(faces.values()) == 2


def test_svd_matches_lapack(oracle_lib):
    rng = np.random.default_rng(0)
    mats = [rng.standard_normal((3, 3)) for _ in range(300)]
    mats += [np.eye(3), np.diag([2.0, 2.0, 1.0]), np.diag([1.0, -1.0, 1.0]), np.zeros((3, 3)),
             np.outer([1.0, 2, 3], [0.5, -1, 2])]
    Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    mats.append(Q)
    mats.append(Q @ np.diag([3.0, 3.0, 3.0]))
    for F in mats:
        U, s, V = oracle_lib.svd3(F)
        assert np.allclose(U @ np.diag(s) @ V.T, F, atol=1e-13)
        assert np.allclose(s, np.linalg.svd(F, compute_uv=False), atol=1e-13)
        assert np.all(s >= 0) and np.all(np.diff(s) <= 0)
        assert np.allclose(U.T @ U, np.eye(3), atol=1e-13)
        assert np.allclose(V.T @ V, np.eye(3), atol=1e-13)


def test_projections(oracle_lib):
    rng = np.random.default_rng(1)
    for _ in range(50):
        F = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        if np.linalg.det(F) <= 0.05:
            continue
        U, s, Vt = np.linalg.svd(F)
        R = oracle_lib.project("corotated", F)
        assert np.allclose(R, U @ Vt, atol=1e-13)
        P = oracle_lib.project("volume", F)
        assert abs(np.linalg.det(P) - 1) < 1e-12
        mu, la = 2e5, 8e5
        k = 2 * mu
        P = oracle_lib.project("pd_neohookean", F, mu, la, k)
        sig = np.linalg.svd(P, compute_uv=False)
        sF = s
        L = np.log(np.prod(sig))
        g = mu * sig - mu / sig + la * L / sig + k * (sig - sF)
        assert np.linalg.norm(g) < 1e-6 * (mu + la)


@pytest.mark.parametrize("kind", ["corotated", "volume", "pd_neohookean"])
def test_projection_differentials(oracle_lib, kind):
    rng = np.random.default_rng(2)
    for _ in range(20):
        F = np.eye(3) + 0.25 * rng.standard_normal((3, 3))
        if np.linalg.det(F) <= 0.1:
            continue
        dF = rng.standard_normal((3, 3))
        args = (1e5, 4e5, 2e5) if kind == "pd_neohookean" else ()
        eps = 1e-6
        a = oracle_lib.project_diff(kind, F, dF, *args)
        b = (oracle_lib.project(kind, F + eps * dF, *args) - oracle_lib.project(kind, F - eps * dF, *args)) / (2 * eps)
        assert np.abs(a - b).max() < 1e-7 * max(1.0, np.abs(a).max())


def test_ainv_matches_dense_solve(oracle_lib):
    sc = scenes.cantilever(cells=(6, 2, 3), steps=1)
    o = oracle_lib.OracleDeformable.from_scene(sc)
    rng = np.random.default_rng(3)
    b = rng.standard_normal(sc.dofs)
    x = o.ainv(b, sc.dt)
    for ax in range(3):
        A = o.dense_A(sc.dt, ax)
        assert np.allclose(A, A.T, atol=1e-9 * np.abs(A).max())
        xr = np.linalg.solve(A, b.reshape(-1, 3)[:, ax])
        assert np.abs(x.reshape(-1, 3)[:, ax] - xr).max() <= 1e-12 * np.abs(xr).max()


def test_rollout_sane(oracle_lib):
    sc = scenes.cantilever(cells=(8, 2, 2), dx=0.02, steps=10)
    o = oracle_lib.OracleDeformable.from_scene(sc)
    q, v, iters = oracle_lib.rollout(o, sc)
    z = q.reshape(-1, 3)[:, 2]
    assert np.all(np.isfinite(q))
    assert z.min() < sc.q0.reshape(-1, 3)[:, 2].min()  # sags under gravity
    fixed = sc.dirichlet_dofs
    assert np.array_equal(q[fixed], sc.dirichlet_vals)


def _adjoint_vs_fd(oracle_lib, sc, eps_v=1e-5):
    opt = dict(sc.options)
    opt.update(rel_tol=1e-12, abs_tol=1e-14, max_pd_iter=4000, aa_window=0)
    r = np.random.default_rng(3).standard_normal(sc.dofs)

    def make(params=None):
        o = oracle_lib.OracleDeformable(sc.verts, sc.elems, sc.density)
        for d, v in zip(sc.dirichlet_dofs, sc.dirichlet_vals):
            o.set_dirichlet(int(d), float(v))
        ens = sc.energies if params is None else [(k, p, i) for (k, _, i), p in zip(sc.energies, params)]
        for k, p, i in ens:
            o.add_pd_energy(k, p, i)
        o.add_gravity(sc.gravity)
        return o

    def loss(v0=None, params=None):
        o = make(params)
        q, v, _, qs, vs = oracle_lib.rollout(o, sc, v0=v0, options=opt, record=True)
        return q @ r, o, qs, vs

    L, o, qs, vs = loss()
    gq, gv = r.copy(), np.zeros(sc.dofs)
    gp = [np.zeros(np.size(p)) for _, p, _ in sc.energies]
    for i in reversed(range(sc.steps)):
        out = o.backward(qs[i], vs[i], sc.f_ext, sc.dt, qs[i + 1], gq, gv, opt)
        gq, gv = out["dl_dq"], out["dl_dv"]
        for a, b in zip(gp, out["dl_dparams"]):
            a += b
    d = np.random.default_rng(5).standard_normal(sc.dofs)
    d[sc.dirichlet_dofs] = 0
    fd = (loss(v0=sc.v0 + eps_v * d)[0] - loss(v0=sc.v0 - eps_v * d)[0]) / (2 * eps_v)
    assert abs(gv @ d - fd) <= 1e-4 * abs(fd) + 1e-12
    p0 = np.asarray(sc.energies[0][1], float)
    dp = np.random.default_rng(6).standard_normal(p0.size) * p0 * 1e-3
    ps = lambda s: [p0 + s * dp] + [np.asarray(p, float) for _, p, _ in sc.energies[1:]]
    fd = (loss(params=ps(1))[0] - loss(params=ps(-1))[0]) / 2
    assert abs(gp[0] @ dp - fd) <= 1e-3 * abs(fd) + 1e-14


def test_adjoint_fd_hex_heterogeneous(oracle_lib):
    _adjoint_vs_fd(oracle_lib, scenes.cantilever(cells=(4, 2, 2), dx=0.02, steps=3, heterogeneous=True))


def test_adjoint_fd_tet_neohookean(oracle_lib):
    _adjoint_vs_fd(oracle_lib, scenes.nh_tet_block(cells=(4, 2, 2), dx=0.01, steps=3))


def test_contact_rollout_stays_above_ground(oracle_lib):
    sc = scenes.contact_drop(cells=(3, 3, 3), dx=0.02, steps=40, height=0.005, friction_mu=0.5)
    o = oracle_lib.OracleDeformable.from_scene(sc)
    opt = dict(sc.options)
    opt["max_pd_iter"] = 300
    q, v, iters = oracle_lib.rollout(o, sc, options=opt)
    z = q.reshape(-1, 3)[:, 2]
    assert np.all(np.isfinite(q))
    assert z.min() > -2e-3          # NCP keeps the nodes (approximately) on or above the plane
    assert z.min() < 0.005          # and the block did fall onto it
