"""Python facade over libdiffphd_b200.so, mirroring the reference's SWIG `HexDeformable` / `TetDeformable`
(cpp/core/src/py_diff_pd_core.i:60-68; method names from cpp/core/include/fem/deformable.h) so that code
written against `py_diff_pd` (e.g. python/py_diff_pd/env/env_base.py:163-427) runs unchanged on the B200
path.  Vectors may be lists, numpy arrays or the `StdRealVector` / `StdIntVector` helpers; outputs are
written into the mutable containers passed in, as SWIG's by-reference std::vector outputs are.

The computation always runs in the CUDA library; there is no CPU fallback.  Errors raised by the library
(the reference's CheckError) surface as RuntimeError with the library's message.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libdiffphd_b200.so"
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


class StdRealVector(list):
    """Stand-in for the reference's SWIG StdRealVector (a resizable list of floats)."""

    def __init__(self, n=0):
        super().__init__([0.0] * int(n) if isinstance(n, (int, np.integer)) else list(n))


class StdIntVector(list):
    def __init__(self, n=0):
        super().__init__([0] * int(n) if isinstance(n, (int, np.integer)) else list(n))


def load_library():
    """Load the in-tree CUDA library; fails loudly when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"diffphd_b200 CUDA library missing at {LIB_PATH}; build it with "
                           "`python -m diffphd_b200.build` (there is no CPU fallback)")
    L = C.CDLL(str(LIB_PATH))
    L.dphd_last_error.restype = C.c_char_p
    L.dphd_create.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    L.dphd_destroy.argtypes = [C.c_void_p]
    L.dphd_init_from_bin.argtypes = [C.c_void_p, C.c_char_p, C.c_double, C.c_char_p, C.c_double, C.c_double]
    L.dphd_init_from_arrays.argtypes = [C.c_void_p, _dp, C.c_int, _ip, C.c_int, C.c_double, C.c_char_p, C.c_double,
                                        C.c_double]
    L.dphd_set_dirichlet.argtypes = [C.c_void_p, C.c_int, C.c_double]
    L.dphd_add_pd_energy.argtypes = [C.c_void_p, C.c_char_p, _dp, C.c_int, _ip, C.c_int]
    L.dphd_add_state_force.argtypes = [C.c_void_p, C.c_char_p, _dp, C.c_int]
    L.dphd_set_frictional_boundary.argtypes = [C.c_void_p, C.c_char_p, _dp, C.c_int, _ip, C.c_int]
    for f in ("dphd_dofs", "dphd_act_dofs", "dphd_num_pd_element_energies", "dphd_num_state_force_parameters",
              "dphd_num_pd_params", "dphd_num_frames", "dphd_last_backward_iters"):
        getattr(L, f).argtypes = [C.c_void_p]
    L.dphd_s_memory_bytes.argtypes = [C.c_void_p]
    L.dphd_s_memory_bytes.restype = C.c_longlong
    L.dphd_s_nnz.argtypes = [C.c_void_p]
    L.dphd_s_nnz.restype = C.c_longlong
    L.dphd_frame_stats.argtypes = [C.c_void_p, _ip, _ip]
    L.dphd_reset_frame_stats.argtypes = [C.c_void_p]
    kv = [C.POINTER(C.c_char_p), _dp, C.c_int]
    L.dphd_forward.argtypes = [C.c_void_p, C.c_char_p, _dp, _dp, _dp, _dp, C.c_double] + kv + [_dp, _dp, _ip, _ip]
    bw = [C.c_void_p, C.c_char_p, _dp, _dp, _dp, _dp, C.c_double, _dp, _dp, _ip, C.c_int, _dp, _dp] + kv + \
         [_dp, _dp, _dp, _dp, _dp, _dp, _dp]
    L.dphd_backward.argtypes = bw
    L.dphd_backward_ex.argtypes = bw + [_dp]
    L.dphd_forward_device.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double] + kv + \
                                     [C.c_void_p, C.c_void_p, C.c_void_p]
    L.dphd_backward_device.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double] + \
        kv + [C.c_void_p] * 7
    L.dphd_reset_warm_start.argtypes = [C.c_void_p]
    L.dphd_kernel_launches.argtypes = [C.c_void_p]
    L.dphd_kernel_launches.restype = C.c_longlong
    L.dphd_device.argtypes = [C.c_void_p]
    L.dphd_debug_set_st_schedule.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.dphd_contact_path_stats.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                          C.POINTER(C.c_int)]
    L.dphd_debug_set_mma_wait_polls.argtypes = [C.c_longlong]
    L.dphd_fp64_escalations.argtypes = [C.c_void_p]
    L.dphd_ncp_solve_stats.argtypes = [C.c_void_p] + [C.POINTER(C.c_longlong)] * 4
    L.dphd_warm_start_state.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_void_p]
    L.dphd_backward_fallbacks.argtypes = [C.c_void_p]
    L.dphd_debug_set_factor_build.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.dphd_factor_built_on_device.argtypes = [C.c_void_p]
    L.dphd_s_padded_values.argtypes = [C.c_void_p]
    L.dphd_s_padded_values.restype = C.c_longlong
    L.dphd_debug_time_ainv.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int, _dp]
    L.dphd_ainv_noalloc.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    L.dphd_debug_ainv.argtypes = [C.c_void_p, C.c_double, _dp, _dp, C.c_int]
    L.dphd_forward_device_init.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_double] + kv + [C.c_void_p] * 4
    L.dphd_mlp_sizes.argtypes = [_ip, _ip, _ip, _ip]
    L.dphd_set_warm_start_network.argtypes = [C.c_void_p] * 3
    L.dphd_contact_adjoint_stats.argtypes = [C.c_void_p, _ip, _ip, _ip]
    L.dphd_last_filtered_samples.argtypes = [C.c_void_p]
    L.dphd_num_contact_candidates.argtypes = [C.c_void_p]
    L.dphd_contact_lambda_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    L.dphd_mlp_pack.argtypes = [C.c_void_p] * 3
    L.dphd_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.dphd_mlp_forward_tc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
    L.dphd_mlp_train_step.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_void_p] + [C.c_float] * 5 + \
        [C.c_int] + [C.c_void_p] * 5
    L.dphd_warmstart_features.argtypes = [C.c_void_p, C.c_double] + [C.c_void_p] * 8
    L.dphd_warmstart_apply.argtypes = [C.c_void_p, C.c_double] + [C.c_void_p] * 4
    L.dphd_warmstart_target.argtypes = [C.c_void_p, C.c_double] + [C.c_void_p] * 4
    L.dphd_debug_host_sts.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
    L.dphd_debug_s_rows.argtypes = [C.c_void_p, C.c_double, _ip, _ip]
    L.dphd_debug_set_s_kernel.argtypes = [C.c_void_p, C.c_int]
    L.dphd_debug_set_pdl.argtypes = [C.c_void_p, C.c_int]
    L.dphd_debug_local_step.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
    _lib = L
    return L


def exported_symbols():
    """Names declared in include/diffphd_b200.h (for the ABI completeness test)."""
    import re
    hdr = (_PKG.parent / "include" / "diffphd_b200.h").read_text()
    return sorted(set(re.findall(r"\b(dphd_[a-z_0-9]+)\s*\(", hdr)))


def _arr(x, n=None):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())
    if n is not None and a.size != n:
        raise RuntimeError(f"Inconsistent vector size: expected {n}, got {a.size}")
    return a


def _iarr(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.int32).ravel())


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _iptr(a):
    return a.ctypes.data_as(_ip)


def _opts(options):
    options = dict(options or {})
    keys = [str(k) for k in options]
    karr = (C.c_char_p * max(1, len(keys)))(*[k.encode() for k in keys])
    vals = np.array([float(options[k]) for k in keys] or [0.0], dtype=np.float64)
    return karr, vals, len(keys)


def _write_out(dst, src):
    """Copy into a by-reference output: numpy array in place, list-likes resized."""
    if isinstance(dst, np.ndarray):
        dst.reshape(-1)[:] = src
    elif isinstance(dst, list):
        dst[:] = list(src)
    elif dst is not None:
        raise TypeError("output containers must be numpy arrays or lists")


class Deformable:
    vertex_dim = 3
    element_dim = 8

    def __init__(self):
        L = load_library()
        h = C.c_void_p()
        self._check(L.dphd_create(3, self.element_dim, C.byref(h)))
        self._h = h
        self._L = L

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_L", None) is not None:
            self._L.dphd_destroy(h)
            self._h = None

    @staticmethod
    def _check(rc):
        if rc != 0:
            raise RuntimeError(load_library().dphd_last_error().decode())

    # ---- builder --------------------------------------------------------------------------------
    def Initialize(self, mesh_or_vertices, *args):
        """Initialize(bin_file, density, material_type, E, nu) or
        Initialize(vertices (n,3), elements (m,k), density, material_type, E, nu)."""
        if isinstance(mesh_or_vertices, (str, os.PathLike)):
            density, material, E, nu = args
            self._check(self._L.dphd_init_from_bin(self._h, str(mesh_or_vertices).encode(), float(density),
                                                   material.encode(), float(E), float(nu)))
        else:
            elements, density, material, E, nu = args
            v = _arr(mesh_or_vertices)
            e = _iarr(elements)
            self._check(self._L.dphd_init_from_arrays(self._h, _ptr(v), v.size // 3, _iptr(e),
                                                      e.size // self.element_dim, float(density), material.encode(),
                                                      float(E), float(nu)))

    def SetDirichletBoundaryCondition(self, dof, val):
        self._check(self._L.dphd_set_dirichlet(self._h, int(dof), float(val)))

    def AddPdEnergy(self, energy_type, params, indices):
        p = _arr(params)
        i = _iarr(indices)
        self._check(self._L.dphd_add_pd_energy(self._h, energy_type.encode(), _ptr(p), p.size, _iptr(i), i.size))

    def AddStateForce(self, force_type, params):
        p = _arr(params)
        self._check(self._L.dphd_add_state_force(self._h, force_type.encode(), _ptr(p), p.size))

    def SetFrictionalBoundary(self, boundary_type, params, indices):
        p = _arr(params)
        i = _iarr(indices)
        self._check(self._L.dphd_set_frictional_boundary(self._h, boundary_type.encode(), _ptr(p), p.size,
                                                         _iptr(i), i.size))

    # ---- accessors ------------------------------------------------------------------------------
    def dofs(self):
        return self._L.dphd_dofs(self._h)

    def act_dofs(self):
        return self._L.dphd_act_dofs(self._h)

    def NumOfPdElementEnergies(self):
        return self._L.dphd_num_pd_element_energies(self._h)

    def NumOfPdMuscleEnergies(self):
        return 0

    def NumOfStateForceParameters(self):
        return self._L.dphd_num_state_force_parameters(self._h)

    def NumOfPdParams(self):
        return self._L.dphd_num_pd_params(self._h)

    # ---- step ------------------------------------------------------------------------------------
    def PyForward(self, method, q, v, a, f_ext, dt, options, q_next, v_next, active_contact_idx):
        n = self.dofs()
        qa, va, fa = _arr(q, n), _arr(v, n), _arr(f_ext, n)
        aa = _arr(a) if a is not None and len(a) else np.zeros(1)
        qn, vn = np.zeros(n), np.zeros(n)
        act = np.zeros(max(1, n // 3), dtype=np.int32)
        na = C.c_int(act.size)
        k, vals, no = _opts(options)
        self._check(self._L.dphd_forward(self._h, method.encode(), _ptr(qa), _ptr(va), _ptr(aa), _ptr(fa),
                                         float(dt), k, _ptr(vals), no, _ptr(qn), _ptr(vn), _iptr(act),
                                         C.byref(na)))
        _write_out(q_next, qn)
        _write_out(v_next, vn)
        if active_contact_idx is not None:
            _write_out(active_contact_idx, act[:na.value].tolist() if isinstance(active_contact_idx, list)
                       else act[:na.value])
        return qn, vn

    def PyBackward(self, method, q, v, a, f_ext, dt, q_next, v_next, active_contact_idx, dl_dq_next, dl_dv_next,
                   options, dl_dq, dl_dv, dl_da, dl_df_ext, dl_dmat_w, dl_dact_w, dl_dstate_p):
        out = self.backward(method, q, v, a, f_ext, dt, q_next, v_next, active_contact_idx, dl_dq_next,
                            dl_dv_next, options)
        for dst, key in ((dl_dq, "dl_dq"), (dl_dv, "dl_dv"), (dl_da, "dl_da"), (dl_df_ext, "dl_df_ext"),
                         (dl_dmat_w, "dl_dmat_w"), (dl_dact_w, "dl_dact_w"), (dl_dstate_p, "dl_dstate_p")):
            _write_out(dst, out[key])
        return out

    def backward(self, method, q, v, a, f_ext, dt, q_next, v_next, active_contact_idx, dl_dq_next, dl_dv_next,
                 options):
        """PyBackward returning a dict, with the extension `dl_dparams` (per AddPdEnergy parameter arrays)."""
        n = self.dofs()
        arrs = [_arr(x, n) for x in (q, v, f_ext, q_next, v_next, dl_dq_next, dl_dv_next)]
        qa, va, fa, qna, vna, g1, g2 = arrs
        aa = _arr(a) if a is not None and len(a) else np.zeros(1)
        act = _iarr(active_contact_idx if active_contact_idx is not None else [])
        actp = act if act.size else np.zeros(1, np.int32)
        dq, dv, df = np.zeros(n), np.zeros(n), np.zeros(n)
        ne = self.NumOfPdElementEnergies()
        ns = self.NumOfStateForceParameters()
        npar = self.NumOfPdParams()
        dmat, dstate, dpar = np.zeros(max(ne, 1)), np.zeros(max(ns, 1)), np.zeros(max(npar, 1))
        da, dact = np.zeros(1), np.zeros(1)
        k, vals, no = _opts(options)
        self._check(self._L.dphd_backward_ex(self._h, method.encode(), _ptr(qa), _ptr(va), _ptr(aa), _ptr(fa),
                                             float(dt), _ptr(qna), _ptr(vna), _iptr(actp), int(act.size), _ptr(g1),
                                             _ptr(g2), k, _ptr(vals), no, _ptr(dq), _ptr(dv), _ptr(da), _ptr(df),
                                             _ptr(dmat), _ptr(dact), _ptr(dstate), _ptr(dpar)))
        return {"dl_dq": dq, "dl_dv": dv, "dl_da": np.zeros(self.act_dofs()), "dl_df_ext": df,
                "dl_dmat_w": dmat[:ne], "dl_dact_w": np.zeros(0), "dl_dstate_p": dstate[:ns],
                "dl_dparams": dpar[:npar], "iters": self._L.dphd_last_backward_iters(self._h)}

    def forward_device(self, method, q, v, f_ext, dt, options, q_next, v_next, stream=0):
        """Device-pointer step on torch CUDA tensors (float64, contiguous, 3n); `stream` is a raw cudaStream_t."""
        k, vals, no = _opts(options)
        self._check(self._L.dphd_forward_device(self._h, method.encode(), C.c_void_p(q.data_ptr()),
                                                C.c_void_p(v.data_ptr()), C.c_void_p(f_ext.data_ptr()), float(dt),
                                                k, _ptr(vals), no, C.c_void_p(q_next.data_ptr()),
                                                C.c_void_p(v_next.data_ptr()), C.c_void_p(int(stream))))

    def forward_device_init(self, method, q, v, f_ext, dt, options, q_init, q_next, v_next, stream=0):
        """forward_device whose PD loop starts from q_init (3n float64 CUDA tensor) instead of q."""
        k, vals, no = _opts(options)
        ptr = lambda t: C.c_void_p(t.data_ptr())
        self._check(self._L.dphd_forward_device_init(self._h, method.encode(), ptr(q), ptr(v), ptr(f_ext), float(dt),
                                                     k, _ptr(vals), no, ptr(q_init), ptr(q_next), ptr(v_next),
                                                     C.c_void_p(int(stream))))

    def set_warm_start_network(self, mlp):
        """Attach a trained `warmstart.WarmStartMLP` (its weights are copied) or detach it (None): while
        attached, PyForward / forward_device start each PD loop from the network's prediction."""
        if mlp is None:
            self._check(self._L.dphd_set_warm_start_network(self._h, None, None))
        else:
            import torch
            torch.cuda.synchronize(mlp.device)  # the weights may still be in flight on a torch stream
            self._check(self._L.dphd_set_warm_start_network(self._h, C.c_void_p(mlp.master.data_ptr()),
                                                            C.c_void_p(mlp.packed.data_ptr())))

    def warmstart_features(self, dt, q, q_prev, v, f_ext, prev_base, X, base, stream=0):
        ptr = lambda t: C.c_void_p(t.data_ptr() if t is not None else 0)
        self._check(self._L.dphd_warmstart_features(self._h, float(dt), ptr(q), ptr(q_prev), ptr(v), ptr(f_ext),
                                                    ptr(prev_base), ptr(X), ptr(base), C.c_void_p(int(stream))))

    def warmstart_apply(self, dt, base, out, q_init, stream=0):
        ptr = lambda t: C.c_void_p(t.data_ptr())
        self._check(self._L.dphd_warmstart_apply(self._h, float(dt), ptr(base), ptr(out), ptr(q_init),
                                                 C.c_void_p(int(stream))))

    def warmstart_target(self, dt, q_next, base, Y, stream=0):
        ptr = lambda t: C.c_void_p(t.data_ptr())
        self._check(self._L.dphd_warmstart_target(self._h, float(dt), ptr(q_next), ptr(base), ptr(Y),
                                                  C.c_void_p(int(stream))))

    def backward_device(self, method, q_next, dl_dq_next, dl_dv_next, dt, options, dl_dq, dl_dv, dl_df_ext,
                        dl_dmat_w=None, dl_dparams=None, dl_dstate_p=None, stream=0):
        """Device-pointer adjoint step on torch CUDA tensors (float64, contiguous)."""
        k, vals, no = _opts(options)
        ptr = lambda t: C.c_void_p(t.data_ptr() if t is not None else 0)
        self._check(self._L.dphd_backward_device(self._h, method.encode(), ptr(q_next), ptr(dl_dq_next),
                                                 ptr(dl_dv_next), float(dt), k, _ptr(vals), no, ptr(dl_dq),
                                                 ptr(dl_dv), ptr(dl_df_ext), ptr(dl_dmat_w), ptr(dl_dparams),
                                                 ptr(dl_dstate_p), C.c_void_p(int(stream))))

    def reset_warm_start(self):
        self._check(self._L.dphd_reset_warm_start(self._h))

    def set_factor_build(self, mode, small_subtree_max=0):
        """0 automatic, 1 host, 2 device construction of the sparse-inverse factor (next build); in device mode the
        etree subtrees of at most `small_subtree_max` nodes (512 when 0) are still built on the host."""
        self._check(self._L.dphd_debug_set_factor_build(self._h, int(mode), int(small_subtree_max)))

    def contact_path_stats(self):
        """(entries, rows of their union, longest path) of the contact candidates' S column paths."""
        e, r, m = C.c_longlong(0), C.c_int(0), C.c_int(0)
        self._check(self._L.dphd_contact_path_stats(self._h, C.byref(e), C.byref(r), C.byref(m)))
        return e.value, r.value, m.value

    def set_st_schedule(self, chunk_rows, rows_in_flight):
        """Schedule of the S^T pass (rows per chunk CTA, rows in flight per warp: 4 or 8) for the next factor build."""
        self._check(self._L.dphd_debug_set_st_schedule(self._h, int(chunk_rows), int(rows_in_flight)))

    def factor_built_on_device(self):
        return int(self._L.dphd_factor_built_on_device(self._h)) == 1

    def warm_start_state(self, stream=0):
        """(valid, 2*3n float64 CUDA tensor): the learned start's previous-step state (for checkpoints)."""
        import torch
        buf = torch.zeros(2 * self.dofs(), dtype=torch.float64, device="cuda")
        valid = C.c_int(0)
        self._check(self._L.dphd_warm_start_state(self._h, C.c_void_p(buf.data_ptr()), C.byref(valid), 0,
                                                  C.c_void_p(int(stream))))
        return valid.value, buf

    def set_warm_start_state(self, state, stream=0):
        valid, buf = state
        v = C.c_int(int(valid))
        self._check(self._L.dphd_warm_start_state(self._h, C.c_void_p(buf.data_ptr()), C.byref(v), 1,
                                                  C.c_void_p(int(stream))))

    def backward_fallbacks(self):
        """Adjoint solves that fell back from CG (to the fixed point, or to the unconstrained adjoint)."""
        return int(self._L.dphd_backward_fallbacks(self._h))

    def ncp_solve_stats(self, detail=False):
        """(solves by the cached factor, refactorisations) of the NCP's dense system since the contact set-up;
        with detail=True also (CG iterations of the cached solves, CG attempts that fell back to a factorisation)."""
        v = [C.c_longlong(0) for _ in range(4)]
        self._check(self._L.dphd_ncp_solve_stats(self._h, *[C.byref(x) for x in v]))
        out = tuple(x.value for x in v)
        return out if detail else out[:2]

    def fp64_escalations(self):
        """Mixed-precision frames that finished in FP64 after the FP32 iteration stalled."""
        return int(self._L.dphd_fp64_escalations(self._h))

    def device(self):
        """CUDA device holding this deformable's GPU state (-1 before the first call that builds it)."""
        return int(self._L.dphd_device(self._h))

    def kernel_launches(self):
        return int(self._L.dphd_kernel_launches(self._h))

    def s_padded_values(self):
        return int(self._L.dphd_s_padded_values(self._h))

    def time_ainv(self, dt, reps=20, fp32=False, flush_l2=True):
        ms = C.c_double(0)
        self._check(self._L.dphd_debug_time_ainv(self._h, float(dt), int(reps), int(bool(fp32)), int(bool(flush_l2)),
                                                 C.byref(ms)))
        return ms.value

    # ---- statistics ------------------------------------------------------------------------------
    def frame_stats(self):
        nf = self._L.dphd_num_frames(self._h)
        it = np.zeros(max(nf, 1), np.int32)
        cv = np.zeros(max(nf, 1), np.int32)
        self._check(self._L.dphd_frame_stats(self._h, _iptr(it), _iptr(cv)))
        return it[:nf].copy(), cv[:nf].copy()

    def num_contact_candidates(self):
        return int(self._L.dphd_num_contact_candidates(self._h))

    def contact_lambda(self, out=None, stream=0):
        """The contact multipliers (lambda warm start) as a float64 CUDA tensor (copied into `out` if given)."""
        import torch
        k = self.num_contact_candidates()
        if out is None:
            out = torch.empty(max(k, 0), dtype=torch.float64, device="cuda")
        if k > 0:
            self._check(self._L.dphd_contact_lambda_device(self._h, C.c_void_p(out.data_ptr()), 0,
                                                           C.c_void_p(int(stream))))
        return out

    def set_contact_lambda(self, lam, stream=0):
        k = self.num_contact_candidates()
        if k > 0:
            if lam.numel() != k or lam.dtype.itemsize != 8 or not lam.is_cuda:
                raise RuntimeError(f"contact multipliers: expected {k} float64 values on the GPU")
            self._check(self._L.dphd_contact_lambda_device(self._h, C.c_void_p(lam.data_ptr()), 1,
                                                           C.c_void_p(int(stream))))

    def last_filtered_samples(self):
        """Samples whose local Hessian the last backward eigen-filtered (option bwd_eigen_filter)."""
        return int(self._L.dphd_last_filtered_samples(self._h))

    def contact_adjoint_stats(self):
        """(source, constraints, cg_iters) of the last backward's contact-aware material adjoint: source 0 none,
        1 forward tape, 2 replayed forward step, 3 tape miss without replay inputs."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._check(self._L.dphd_contact_adjoint_stats(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def reset_frame_stats(self):
        self._check(self._L.dphd_reset_frame_stats(self._h))

    def s_memory_bytes(self):
        return int(self._L.dphd_s_memory_bytes(self._h))

    def s_nnz(self):
        return int(self._L.dphd_s_nnz(self._h))

    # ---- diagnostics -----------------------------------------------------------------------------
    def debug_s_rows(self, dt):
        """(lo, perm): first column of each row of the sparse inverse factor S and the permutation (host only)."""
        n = self.dofs() // 3
        lo, perm = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self._check(self._L.dphd_debug_s_rows(self._h, float(dt), _iptr(lo), _iptr(perm)))
        return lo, perm

    def set_pdl(self, on=True):
        """Programmatic dependent launch of the iteration-body kernels (process-wide; default on)."""
        self._check(self._L.dphd_debug_set_pdl(self._h, int(bool(on))))

    def set_s_kernel(self, row_groups=True):
        """FP32 y = S v pass: one warp per row group or one warp per row segment (bit-identical sums; by default
        the faster one is picked by timing both when the factor is built)."""
        self._check(self._L.dphd_debug_set_s_kernel(self._h, int(bool(row_groups))))

    def debug_ainv(self, b, dt, fp32=False):
        b = _arr(b, self.dofs())
        x = np.zeros_like(b)
        self._check(self._L.dphd_debug_ainv(self._h, float(dt), _ptr(b), _ptr(x), int(bool(fp32))))
        return x

    def debug_host_sts(self, b, dt):
        b = _arr(b, self.dofs())
        x = np.zeros_like(b)
        self._check(self._L.dphd_debug_host_sts(self._h, float(dt), _ptr(b), _ptr(x)))
        return x

    def debug_local_step(self, q, dt):
        q = _arr(q, self.dofs())
        r = np.zeros_like(q)
        self._check(self._L.dphd_debug_local_step(self._h, float(dt), _ptr(q), _ptr(r)))
        return r


class HexDeformable(Deformable):
    element_dim = 8


class TetDeformable(Deformable):
    element_dim = 4


def from_scene(scene):
    """Build a Hex/TetDeformable from a diffphd_b200.scenes.Scene with the reference builder calls."""
    cls = HexDeformable if scene.elems.shape[1] == 8 else TetDeformable
    d = cls()
    d.Initialize(scene.verts, scene.elems, scene.density, "none", 0.0, 0.0)
    for dof, val in zip(scene.dirichlet_dofs, scene.dirichlet_vals):
        d.SetDirichletBoundaryCondition(int(dof), float(val))
    for kind, params, idx in scene.energies:
        d.AddPdEnergy(kind, params, idx)
    if scene.gravity is not None:
        d.AddStateForce("gravity", scene.gravity)
    if scene.plane is not None:
        d.SetFrictionalBoundary("planar", scene.plane[0], scene.plane[1])
    return d
