"""Seeded synthetic scenes for the projective-dynamics step (no datasets are involved).

Each builder returns a `Scene`: the mesh, material and boundary set-up expressed in the
reference's builder vocabulary (`AddPdEnergy`, `SetDirichletBoundaryCondition`,
`AddStateForce('gravity')`, `SetFrictionalBoundary('planar')`), the step size, rollout length,
solver options and initial state.  The same description feeds the CUDA path and the CPU oracle.

Scenes (sizes are what they are named for):
  * cantilever_hex_16x4x4  — 425 nodes, corotated + volume, x=0 face clamped, gravity, dt 1e-2.
    Mirrors python/py_diff_pd/env/cantilever_env_3d.py:19-59 (material 'none', per-energy PD weights).
  * nh_tet_block_32x16x16  — 32x16x16 cells split into 5 tets each (40,960 tets, 9,537 nodes),
    per-element Neo-Hookean (mu_e, lambda_e) from a seeded two-phase blob field (1e5 / 1e7 Pa,
    blob radius 3 cells), nu 0.45, x=0 end clamped, gravity, dt 5e-3.
  * contact_drop_hex_24    — 24^3 hex block, corotated E 5e5 nu 0.4, seeded rotation, dropped from
    0.05 m onto z=0 with Coulomb mu 0.5, every node a contact candidate, dt 5e-3.
  * hetero_contact_hex_64  — 64^3 hex block, lognormal E_e, uniform nu_e, ground contact mu 0.3, dt 2e-3.
All take a `cells` override so tests can run the same physics on smaller grids.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .mesh import generate_hex_mesh, hex_to_tet5


def lame(E, nu):
    E = np.asarray(E, dtype=np.float64)
    nu = np.asarray(nu, dtype=np.float64)
    mu = E / (2 * (1 + nu))
    la = E * nu / ((1 + nu) * (1 - 2 * nu))
    return mu, la


def lame_jacobian(E, nu):
    """d(mu, la)/d(E, nu), elementwise: returns (dmu_dE, dmu_dnu, dla_dE, dla_dnu)."""
    E = np.asarray(E, dtype=np.float64)
    nu = np.asarray(nu, dtype=np.float64)
    dmu_dE = 1 / (2 * (1 + nu))
    dmu_dnu = -E / (2 * (1 + nu) ** 2)
    den = (1 + nu) * (1 - 2 * nu)
    dla_dE = nu / den
    dla_dnu = E * (1 + 2 * nu ** 2) / den ** 2
    return dmu_dE, dmu_dnu, dla_dE, dla_dnu


@dataclass
class Scene:
    name: str
    verts: np.ndarray            # (n, 3) rest positions
    elems: np.ndarray            # (m, k) connectivity
    density: float
    energies: list               # [(type, params ndarray, element index list)]
    dirichlet_dofs: np.ndarray
    dirichlet_vals: np.ndarray
    gravity: np.ndarray | None
    plane: tuple | None          # ((nx, ny, nz, offset), node indices)
    dt: float
    steps: int
    options: dict
    q0: np.ndarray
    v0: np.ndarray
    f_ext: np.ndarray
    youngs: np.ndarray | None = None      # per-element E (for chaining parameter gradients)
    poisson: np.ndarray | None = None
    material_kind: str = "corotated"     # 'corotated' (corotated+volume) or 'pd_neohookean'
    extra: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.verts.shape[0]

    @property
    def m(self):
        return self.elems.shape[0]

    @property
    def dofs(self):
        return 3 * self.n


def default_options(rel_tol=1e-6, abs_tol=1e-9, max_pd_iter=500, thread_ct=8, aa_window=5):
    return {"max_pd_iter": max_pd_iter, "abs_tol": abs_tol, "rel_tol": rel_tol, "verbose": 0,
            "thread_ct": thread_ct, "aa_window": aa_window}


def _clamp_face(verts, axis=0, value=None):
    v = verts[:, axis]
    value = v.min() if value is None else value
    nodes = np.nonzero(np.abs(v - value) < 1e-12)[0]
    dofs = (3 * nodes[:, None] + np.arange(3)[None, :]).ravel()
    vals = verts[nodes].ravel()
    return dofs.astype(np.int64), vals.astype(np.float64)


def cantilever(cells=(16, 4, 4), dx=0.01, E=1e6, nu=0.45, density=1e3, dt=1e-2, steps=100, seed=0,
               options=None, heterogeneous=False):
    verts, hexes, _ = generate_hex_mesh(np.ones(cells), dx)
    mu, la = lame(E, nu)
    m = hexes.shape[0]
    if heterogeneous:
        rng = np.random.default_rng(seed + 1)
        Ee = E * np.exp(rng.normal(0.0, 0.5, size=m))
        nue = np.full(m, nu)
        mue, lae = lame(Ee, nue)
        energies = [("corotated", 2 * mue, []), ("volume", lae, [])]
    else:
        Ee = np.full(m, E)
        nue = np.full(m, nu)
        energies = [("corotated", np.array([2 * mu]), []), ("volume", np.array([la]), [])]
    dd, dv = _clamp_face(verts, 0)
    rng = np.random.default_rng(seed)
    n = verts.shape[0]
    return Scene(name="cantilever_hex_%dx%dx%d" % tuple(cells), verts=verts, elems=hexes, density=density,
                 energies=energies, dirichlet_dofs=dd, dirichlet_vals=dv, gravity=np.array([0.0, 0.0, -9.81]),
                 plane=None, dt=dt, steps=steps, options=options or default_options(),
                 q0=verts.ravel().copy(), v0=np.zeros(3 * n), f_ext=np.zeros(3 * n), youngs=Ee, poisson=nue,
                 material_kind="corotated", extra={"loss_r": rng.standard_normal(3 * n)})


def blob_field(cells, radius=3, n_blobs=None, seed=0, soft=1e5, stiff=1e7):
    rng = np.random.default_rng(seed)
    cx, cy, cz = cells
    if n_blobs is None:
        n_blobs = max(1, int(round(cx * cy * cz / (4.0 / 3.0 * np.pi * radius ** 3) * 0.3)))
    centres = rng.uniform([0, 0, 0], [cx, cy, cz], size=(n_blobs, 3))
    I, J, K = np.meshgrid(np.arange(cx) + 0.5, np.arange(cy) + 0.5, np.arange(cz) + 0.5, indexing="ij")
    cc = np.stack([I, J, K], axis=-1)
    inside = np.zeros(cells, dtype=bool)
    for c in centres:
        inside |= np.sum((cc - c) ** 2, axis=-1) <= radius ** 2
    return np.where(inside, stiff, soft)


def nh_tet_block(cells=(32, 16, 16), dx=0.005, nu=0.45, density=1e3, dt=5e-3, steps=200, seed=0, options=None):
    verts, hexes, ijk = generate_hex_mesh(np.ones(cells), dx)
    tets = hex_to_tet5(verts, hexes, ijk)
    field_E = blob_field(cells, radius=3, seed=seed)
    Ee = np.repeat(field_E[ijk[:, 0], ijk[:, 1], ijk[:, 2]], 5)
    nue = np.full(tets.shape[0], nu)
    mue, lae = lame(Ee, nue)
    params = np.stack([mue, lae], axis=1).ravel()
    dd, dv = _clamp_face(verts, 0)
    n = verts.shape[0]
    rng = np.random.default_rng(seed + 7)
    return Scene(name="nh_tet_block_%dx%dx%d" % tuple(cells), verts=verts, elems=tets, density=density,
                 energies=[("pd_neohookean", params, [])], dirichlet_dofs=dd, dirichlet_vals=dv,
                 gravity=np.array([0.0, 0.0, -9.81]), plane=None, dt=dt, steps=steps,
                 options=options or default_options(), q0=verts.ravel().copy(), v0=np.zeros(3 * n),
                 f_ext=np.zeros(3 * n), youngs=Ee, poisson=nue, material_kind="pd_neohookean",
                 extra={"loss_r": rng.standard_normal(3 * n)})


def random_rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def contact_drop(cells=(24, 24, 24), dx=0.01, E=5e5, nu=0.4, density=1e3, dt=5e-3, steps=300, seed=0,
                 friction_mu=0.5, height=0.05, rotate=True, options=None):
    verts, hexes, _ = generate_hex_mesh(np.ones(cells), dx)
    rng = np.random.default_rng(seed)
    q0 = verts.copy()
    if rotate:
        R = random_rotation(rng)
        c = q0.mean(axis=0)
        q0 = (q0 - c) @ R.T + c
    q0[:, 2] += height - q0[:, 2].min()
    mu, la = lame(E, nu)
    m = hexes.shape[0]
    n = verts.shape[0]
    opts = options or default_options()
    opts = dict(opts)
    opts["friction_mu"] = friction_mu
    return Scene(name="contact_drop_hex_%dx%dx%d" % tuple(cells), verts=verts, elems=hexes, density=density,
                 energies=[("corotated", np.array([2 * mu]), []), ("volume", np.array([la]), [])],
                 dirichlet_dofs=np.zeros(0, np.int64), dirichlet_vals=np.zeros(0),
                 gravity=np.array([0.0, 0.0, -9.81]), plane=((0.0, 0.0, 1.0, 0.0), np.arange(n)),
                 dt=dt, steps=steps, options=opts, q0=q0.ravel(), v0=np.zeros(3 * n), f_ext=np.zeros(3 * n),
                 youngs=np.full(m, E), poisson=np.full(m, nu), material_kind="corotated",
                 extra={"loss_r": rng.standard_normal(3 * n)})


def hetero_contact(cells=(64, 64, 64), dx=0.005, density=1e3, dt=2e-3, steps=50, seed=0, friction_mu=0.3,
                   height=0.005, options=None):
    verts, hexes, _ = generate_hex_mesh(np.ones(cells), dx)
    rng = np.random.default_rng(seed)
    m = hexes.shape[0]
    n = verts.shape[0]
    Ee = np.exp(rng.normal(np.log(1e6), 1.0, size=m))
    nue = rng.uniform(0.3, 0.45, size=m)
    mue, lae = lame(Ee, nue)
    q0 = verts.copy()
    q0[:, 2] += height - q0[:, 2].min()
    bottom = np.nonzero(np.abs(verts[:, 2] - verts[:, 2].min()) < 1e-12)[0]
    opts = dict(options or default_options())
    opts["friction_mu"] = friction_mu
    # seeded smooth target displacement field
    k = rng.standard_normal((3, 3)) * 0.01
    target = q0 + np.sin(verts @ k.T * 10.0) * 0.002
    return Scene(name="hetero_contact_hex_%dx%dx%d" % tuple(cells), verts=verts, elems=hexes, density=density,
                 energies=[("corotated", 2 * mue, []), ("volume", lae, [])],
                 dirichlet_dofs=np.zeros(0, np.int64), dirichlet_vals=np.zeros(0),
                 gravity=np.array([0.0, 0.0, -9.81]), plane=((0.0, 0.0, 1.0, 0.0), bottom),
                 dt=dt, steps=steps, options=opts, q0=q0.ravel(), v0=np.zeros(3 * n), f_ext=np.zeros(3 * n),
                 youngs=Ee, poisson=nue, material_kind="corotated", extra={"q_target": target.ravel()})


def energy_params_from_material(scene: Scene, youngs=None, poisson=None):
    """Rebuild the AddPdEnergy parameter arrays of a per-element scene from (E_e, nu_e)."""
    E = scene.youngs if youngs is None else youngs
    nu = scene.poisson if poisson is None else poisson
    mu, la = lame(E, nu)
    if scene.material_kind == "pd_neohookean":
        return [("pd_neohookean", np.stack([mu, la], axis=1).ravel(), [])]
    return [("corotated", 2 * mu, []), ("volume", la, [])]


def chain_material_grad(scene: Scene, dl_dparams_per_energy):
    """Per-element (dl/dE_e, dl/dnu_e) from per-element energy parameter gradients."""
    dmu_dE, dmu_dnu, dla_dE, dla_dnu = lame_jacobian(scene.youngs, scene.poisson)
    if scene.material_kind == "pd_neohookean":
        g = np.asarray(dl_dparams_per_energy[0]).reshape(-1, 2)
        gmu, gla = g[:, 0], g[:, 1]
    else:
        gmu = 2 * np.asarray(dl_dparams_per_energy[0])
        gla = np.asarray(dl_dparams_per_energy[1])
    return gmu * dmu_dE + gla * dla_dE, gmu * dmu_dnu + gla * dla_dnu
