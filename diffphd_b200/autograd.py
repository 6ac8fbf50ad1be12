"""Differentiable rollouts: a torch.autograd.Function over the B200 projective-dynamics step.

The reference wraps PyForward/PyBackward in `SimFunction` (python/py_diff_pd/common/sim.py:9-74), which is
stale (it passes 5 outputs to the 7-output PyBackward).  `Rollout` replaces it for whole rollouts:

    q_T, v_T = Rollout.apply(sim, q0, v0, params, f_ext, steps, checkpoint_every)

* `sim` is a `DiffSim` (scene + options); `params` is the concatenation of every AddPdEnergy parameter
  array (per-element stiffnesses or interleaved [mu_e, la_e]); changing it rebuilds the deformable.
* `f_ext` is one (3n,) external force applied at every step.
* Forward runs on the device entry points and stores (q, v, contact multipliers) every `checkpoint_every`
  steps; backward recomputes each segment from its checkpoint and runs the adjoint through it in reverse
  (the recomputed frames also refill the contact tape that the adjoint pops)
  (forward checkpointing with recomputation; memory is O(T / k + k) states instead of O(T)).
Gradients: q0, v0, params (summed over steps) and f_ext (summed over steps).
"""
from __future__ import annotations

import numpy as np
import torch

from . import core


class DiffSim:
    """A scene whose PD energy parameters can be replaced by a tensor (per-element materials)."""

    def __init__(self, scene, options=None, method="pd_eigen_alg_phd", warm_start_network=None):
        self.scene = scene
        self.options = dict(options or scene.options)
        self.method = method
        self.warm_start_network = warm_start_network  # attached to every deformable this object builds
        self._d = None
        self._params = None
        self.sizes = [int(np.size(p)) for _, p, _ in scene.energies]

    def default_params(self):
        return torch.as_tensor(np.concatenate([np.atleast_1d(np.asarray(p, float)) for _, p, _ in self.scene.energies]))

    def deformable(self, params: np.ndarray):
        if self._d is not None and self._params is not None and np.array_equal(self._params, params):
            return self._d
        sc = self.scene
        cls = core.HexDeformable if sc.elems.shape[1] == 8 else core.TetDeformable
        d = cls()
        d.Initialize(sc.verts, sc.elems, sc.density, "none", 0.0, 0.0)
        for dof, val in zip(sc.dirichlet_dofs, sc.dirichlet_vals):
            d.SetDirichletBoundaryCondition(int(dof), float(val))
        for (kind, _, idx), p in zip(sc.energies, np.split(params, np.cumsum(self.sizes)[:-1])):
            d.AddPdEnergy(kind, p, idx)
        if sc.gravity is not None:
            d.AddStateForce("gravity", sc.gravity)
        if sc.plane is not None:
            d.SetFrictionalBoundary("planar", sc.plane[0], sc.plane[1])
        if self.warm_start_network is not None:
            d.set_warm_start_network(self.warm_start_network)
        self._d, self._params = d, params.copy()
        return d


def _step(d, sim, q, v, f, stream):
    qn, vn = torch.empty_like(q), torch.empty_like(q)
    d.forward_device(sim.method, q, v, f, sim.scene.dt, sim.options, qn, vn, stream=stream)
    return qn, vn


class Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sim: DiffSim, q0, v0, params, f_ext, steps: int, checkpoint_every: int = 10):
        dev = q0.device
        p_np = params.detach().cpu().numpy().astype(np.float64)
        d = sim.deformable(p_np)
        d.reset_warm_start()
        stream = torch.cuda.current_stream(dev).cuda_stream
        q, v = q0.detach().contiguous(), v0.detach().contiguous()
        f = f_ext.detach().contiguous()
        k = max(1, int(checkpoint_every))
        # a checkpoint holds (q, v), the contact multipliers that warm-start the next frame's NCP and the learned
        # start's previous-step state, so that a recomputed segment repeats the forward pass bit for bit
        def snapshot():
            return (q.clone(), v.clone(), d.contact_lambda(stream=stream).clone(), d.warm_start_state(stream=stream))
        ckpts = {0: snapshot()}
        for t in range(steps):
            q, v = _step(d, sim, q, v, f, stream)
            if (t + 1) % k == 0 and t + 1 < steps:
                ckpts[t + 1] = snapshot()
        ctx.sim, ctx.steps, ctx.k, ctx.p_np = sim, steps, k, p_np
        ctx.ckpts = ckpts
        ctx.save_for_backward(f)
        return q.clone(), v.clone()

    @staticmethod
    def backward(ctx, g_q, g_v):
        (f,) = ctx.saved_tensors
        sim, steps, k = ctx.sim, ctx.steps, ctx.k
        d = sim.deformable(ctx.p_np)
        dev = f.device
        stream = torch.cuda.current_stream(dev).cuda_stream
        gq = (g_q if g_q is not None else torch.zeros_like(f)).contiguous().to(torch.float64)
        gv = (g_v if g_v is not None else torch.zeros_like(f)).contiguous().to(torch.float64)
        n_par = d.NumOfPdParams()
        g_par = torch.zeros(max(n_par, 1), dtype=torch.float64, device=dev)
        g_f = torch.zeros_like(f)
        dpar = torch.empty(max(n_par, 1), dtype=torch.float64, device=dev)
        starts = sorted(ctx.ckpts)
        for s in reversed(starts):
            e = min(s + k, steps)
            # recompute the segment's states from its checkpoint (its contact multipliers and learned-start state
            # included); the adjoint history of the later segments is kept: it warm-starts this segment's solves
            q, v, lam, ws = ctx.ckpts[s]
            d.set_contact_lambda(lam, stream=stream)
            d.set_warm_start_state(ws, stream=stream)
            qs = [q]
            for _ in range(s, e):
                q, v = _step(d, sim, q, v, f, stream)
                qs.append(q)
            for t in reversed(range(e - s)):
                dq, dv, df = torch.empty_like(gq), torch.empty_like(gq), torch.empty_like(gq)
                d.backward_device(sim.method, qs[t + 1], gq, gv, sim.scene.dt, sim.options, dq, dv, df,
                                  dl_dparams=dpar, stream=stream)
                gq, gv = dq, dv
                g_par += dpar
                g_f += df
        return None, gq, gv, g_par[:n_par], g_f, None, None
