"""ORACLE — test infrastructure only (ctypes loader for oracle/_build/libpd_oracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module, and only
as the checker.  The product path (diffphd_b200) never imports it.

The oracle is a CPU FP64 restatement of the reference's AlgPhd projective-dynamics step and adjoint
(see oracle/pd_oracle.cpp for the reference files it follows).  Parity against the reference binary
is unpinned: the reference cannot be built here (empty Eigen submodule, no network).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libpd_oracle.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build(quiet=True):
    out = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.orc_last_error.restype = C.c_char_p
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [_dp, C.c_int, _ip, C.c_int, C.c_int, C.c_double]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_dirichlet.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.orc_add_pd_energy.argtypes = [C.c_void_p, C.c_char_p, _dp, C.c_int, _ip, C.c_int]
        L.orc_add_gravity.argtypes = [C.c_void_p, _dp]
        L.orc_set_planar_boundary.argtypes = [C.c_void_p, _dp, _ip, C.c_int]
        L.orc_num_params.argtypes = [C.c_void_p]
        L.orc_mass.argtypes = [C.c_void_p]
        L.orc_mass.restype = C.c_double
        L.orc_last_iters.argtypes = [C.c_void_p]
        L.orc_last_converged.argtypes = [C.c_void_p]
        L.orc_last_filtered.argtypes = [C.c_void_p]
        L.orc_reset_warm_start.argtypes = [C.c_void_p]
        L.orc_forward.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_double, C.POINTER(C.c_char_p), _dp, C.c_int,
                                  _dp, _dp, _ip, _ip]
        L.orc_backward.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_double, _dp, _dp, _dp, C.POINTER(C.c_char_p),
                                   _dp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _ip]
        L.orc_ainv.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
        L.orc_local_step.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_svd3.argtypes = [_dp, _dp, _dp, _dp]
        L.orc_project.argtypes = [C.c_int, _dp, C.c_double, C.c_double, C.c_double, _dp]
        L.orc_project_diff.argtypes = [C.c_int, _dp, C.c_double, C.c_double, C.c_double, _dp, _dp]
        L.orc_dense_A.argtypes = [C.c_void_p, C.c_double, C.c_int, _dp]
        _lib = L
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().orc_last_error().decode())


def _opts(options):
    keys = list(options.keys())
    karr = (C.c_char_p * len(keys))(*[k.encode() for k in keys])
    vals = np.array([float(options[k]) for k in keys], dtype=np.float64)
    return karr, vals, len(keys)


def svd3(F):
    F9 = np.asarray(F, dtype=np.float64).reshape(3, 3).ravel(order="F")
    U = np.zeros(9); s = np.zeros(3); V = np.zeros(9)
    lib().orc_svd3(_d(F9)[1], U.ctypes.data_as(_dp), s.ctypes.data_as(_dp), V.ctypes.data_as(_dp))
    return U.reshape(3, 3, order="F"), s, V.reshape(3, 3, order="F")


TYPES = {"corotated": 0, "volume": 1, "pd_neohookean": 2}


def project(kind, F, mu=0.0, la=0.0, k=0.0):
    F9 = np.asarray(F, dtype=np.float64).reshape(3, 3).ravel(order="F")
    P = np.zeros(9)
    _check(lib().orc_project(TYPES[kind], _d(F9)[1], mu, la, k, P.ctypes.data_as(_dp)))
    return P.reshape(3, 3, order="F")


def project_diff(kind, F, dF, mu=0.0, la=0.0, k=0.0):
    F9 = np.asarray(F, dtype=np.float64).reshape(3, 3).ravel(order="F")
    dF9 = np.asarray(dF, dtype=np.float64).reshape(3, 3).ravel(order="F")
    P = np.zeros(9)
    _check(lib().orc_project_diff(TYPES[kind], _d(F9)[1], mu, la, k, _d(dF9)[1], P.ctypes.data_as(_dp)))
    return P.reshape(3, 3, order="F")


class OracleDeformable:
    """The oracle's model of one scene (mirrors the reference Deformable builder calls)."""

    def __init__(self, verts, elems, density):
        self._keep = []
        v, vp = _d(np.asarray(verts).reshape(-1))
        e, ep = _i(np.asarray(elems).reshape(-1))
        n = np.asarray(verts).reshape(-1, 3).shape[0]
        k = np.asarray(elems).shape[1]
        m = np.asarray(elems).shape[0]
        self.h = lib().orc_create(vp, n, ep, m, k, float(density))
        if not self.h:
            raise RuntimeError(lib().orc_last_error().decode())
        self.n, self.m, self.k = n, m, k
        self.dofs = 3 * n
        self.energy_sizes = []

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    @classmethod
    def from_scene(cls, sc):
        o = cls(sc.verts, sc.elems, sc.density)
        for dof, val in zip(sc.dirichlet_dofs, sc.dirichlet_vals):
            o.set_dirichlet(int(dof), float(val))
        for kind, params, idx in sc.energies:
            o.add_pd_energy(kind, params, idx)
        if sc.gravity is not None:
            o.add_gravity(sc.gravity)
        if sc.plane is not None:
            o.set_planar_boundary(sc.plane[0], sc.plane[1])
        return o

    def set_dirichlet(self, dof, val):
        _check(lib().orc_set_dirichlet(self.h, dof, val))

    def add_pd_energy(self, kind, params, idx=()):
        p, pp = _d(np.atleast_1d(params))
        ix, ip = _i(np.asarray(idx, dtype=np.int32))
        _check(lib().orc_add_pd_energy(self.h, kind.encode(), pp, p.size, ip, ix.size))
        self.energy_sizes.append(p.size)

    def add_gravity(self, g):
        _check(lib().orc_add_gravity(self.h, _d(g)[1]))

    def set_planar_boundary(self, p4, nodes):
        p, pp = _d(p4)
        ix, ip = _i(nodes)
        _check(lib().orc_set_planar_boundary(self.h, pp, ip, ix.size))

    @property
    def mass(self):
        return lib().orc_mass(self.h)

    @property
    def last_iters(self):
        return lib().orc_last_iters(self.h)

    @property
    def last_converged(self):
        """Whether the last forward step's PD loop met its gate before max_pd_iter."""
        return bool(lib().orc_last_converged(self.h))

    @property
    def last_filtered(self):
        """Samples whose Hessian the last backward eigen-filtered (option bwd_eigen_filter)."""
        return lib().orc_last_filtered(self.h)

    def reset_warm_start(self):
        lib().orc_reset_warm_start(self.h)

    def forward(self, q, v, f_ext, dt, options):
        q, qp = _d(q); v, vp = _d(v); f, fp = _d(f_ext)
        qn = np.zeros(self.dofs); vn = np.zeros(self.dofs)
        act = np.zeros(self.n, dtype=np.int32); na = C.c_int(0)
        k, vals, no = _opts(options)
        _check(lib().orc_forward(self.h, qp, vp, fp, dt, k, vals.ctypes.data_as(_dp), no,
                                 qn.ctypes.data_as(_dp), vn.ctypes.data_as(_dp), act.ctypes.data_as(_ip),
                                 C.byref(na)))
        return qn, vn, act[:na.value].copy()

    def backward(self, q, v, f_ext, dt, q_next, dl_dq_next, dl_dv_next, options):
        q, qp = _d(q); v, vp = _d(v); f, fp = _d(f_ext); qn, qnp = _d(q_next)
        g1, g1p = _d(dl_dq_next); g2, g2p = _d(dl_dv_next)
        dq = np.zeros(self.dofs); dv = np.zeros(self.dofs); df = np.zeros(self.dofs)
        nw = len(self.energy_sizes)
        dw = np.zeros(max(nw, 1)); dp = np.zeros(max(lib().orc_num_params(self.h), 1)); ds = np.zeros(3)
        it = C.c_int(0)
        k, vals, no = _opts(options)
        _check(lib().orc_backward(self.h, qp, vp, fp, dt, qnp, g1p, g2p, k, vals.ctypes.data_as(_dp), no,
                                  dq.ctypes.data_as(_dp), dv.ctypes.data_as(_dp), df.ctypes.data_as(_dp),
                                  dw.ctypes.data_as(_dp), dp.ctypes.data_as(_dp), ds.ctypes.data_as(_dp),
                                  C.byref(it)))
        splits = np.cumsum(self.energy_sizes)[:-1]
        return {"dl_dq": dq, "dl_dv": dv, "dl_df_ext": df, "dl_dmat_w": dw[:nw],
                "dl_dparams": np.split(dp[:sum(self.energy_sizes)], splits), "dl_dstate_p": ds,
                "iters": it.value}

    def ainv(self, b, dt):
        b, bp = _d(b)
        x = np.zeros(self.dofs)
        _check(lib().orc_ainv(self.h, dt, bp, x.ctypes.data_as(_dp)))
        return x

    def local_step(self, q):
        q, qp = _d(q)
        r = np.zeros(self.dofs)
        _check(lib().orc_local_step(self.h, qp, r.ctypes.data_as(_dp)))
        return r

    def dense_A(self, dt, axis=0):
        out = np.zeros((self.n, self.n))
        _check(lib().orc_dense_A(self.h, dt, axis, out.ctypes.data_as(_dp)))
        return out


def rollout(o: OracleDeformable, sc, steps=None, q0=None, v0=None, options=None, record=False):
    steps = sc.steps if steps is None else steps
    q = sc.q0.copy() if q0 is None else np.asarray(q0, dtype=np.float64).copy()
    v = sc.v0.copy() if v0 is None else np.asarray(v0, dtype=np.float64).copy()
    opts = sc.options if options is None else options
    qs, vs, iters = [q], [v], []
    o.reset_warm_start()
    for _ in range(steps):
        q, v, _act = o.forward(q, v, sc.f_ext, sc.dt, opts)
        iters.append(o.last_iters)
        if record:
            qs.append(q); vs.append(v)
    return (q, v, iters, qs, vs) if record else (q, v, iters)
