"""Learned warm start of the projective-dynamics fixed point.

The reference starts every PD loop from the current positions q and every NCP from the previous frame's contact
multipliers.  Here a per-node MLP (16 -> 128 -> 128 -> 4, GELU, BF16 tensor-core kernels with FP32 accumulation,
diffphd_b200/csrc/mlp.cu) predicts both: the correction of the inertial prediction
q_tilde = q + h v + h^2/m (f_ext + m g) and, on the contact set, the frame's normal multiplier:

    q_init = q_tilde + dx * MLP(features)[0:3],  lambda_init = max(0, MLP(features)[3]) * m dx / h^2,
    features per node (dphd_warmstart_features):
        (q - X)/dx, (q - q_prev)/dx, (q - q_tilde_prev)/dx, h^2 f_ext/(m dx), height above the contact plane/dx,
        log10(mean PD stiffness)/7, Dirichlet flag, the previous frame's multiplier * h^2/(m dx) (0 off contact)

and the PD loop then runs from q_init to the same dual gate as the plain solver, so the network changes only
the iteration count: a bad prediction costs iterations, never accuracy.  Training data are the plain solver's
own rollouts (targets (q_next - q_tilde)/dx and the frame's final multiplier * h^2/(m dx)); training runs on the GPU through the library's fused training
kernel (forward, backward and weight gradients in one kernel, deterministic AdamW in a second).

    mlp = WarmStartMLP(device, seed=0)
    X, Y = generate_dataset(lambda s: scenes.nh_tet_block(seed=s), seeds=range(20), steps=100, device=dev)
    fit(mlp, X, Y, steps=3000)
    stepper = WarmStartStepper(deformable, mlp, method, dt, options)
    stepper.step(q, v, f_ext, q_next, v_next)
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import core

_p = lambda t: C.c_void_p(t.data_ptr() if t is not None else 0)


def _sizes():
    L = core.load_library()
    a, b, c, d = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    core.Deformable._check(L.dphd_mlp_sizes(C.byref(a), C.byref(b), C.byref(c), C.byref(d)))
    return a.value, b.value, c.value, d.value


N_IN, N_HID, N_OUT, N_USED = 16, 128, 8, 4


class WarmStartMLP:
    """FP32 master weights, BF16 operand copies and AdamW moments, all device tensors owned by torch."""

    def __init__(self, device, seed=0):
        self.device = torch.device(device)
        self.n_master, self.n_packed, self.part_per_block, self.rows_per_block = _sizes()
        g = torch.Generator().manual_seed(int(seed))
        W1 = torch.randn(N_IN, N_HID, generator=g, dtype=torch.float64) * math.sqrt(2.0 / N_IN)
        W2 = torch.randn(N_HID, N_HID, generator=g, dtype=torch.float64) * math.sqrt(2.0 / N_HID)
        W3 = torch.randn(N_HID, N_OUT, generator=g, dtype=torch.float64) * (0.1 / math.sqrt(N_HID))
        W3[:, N_USED:] = 0
        flat = torch.cat([W1.ravel(), W2.ravel(), W3.ravel(), torch.zeros(2 * N_HID + N_OUT, dtype=torch.float64)])
        assert flat.numel() == self.n_master
        self.master = flat.to(torch.float32).to(self.device)
        self.packed = torch.zeros(self.n_packed, dtype=torch.bfloat16, device=self.device)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.step_count = 0
        self.loss_buf = torch.zeros(1, dtype=torch.float32, device=self.device)
        self._part = None
        self._err = None
        self.pack()

    @property
    def _L(self):
        return core.load_library()

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def pack(self):
        core.Deformable._check(self._L.dphd_mlp_pack(_p(self.master), _p(self.packed), self._stream()))

    def load_master(self, flat):
        self.master.copy_(torch.as_tensor(flat, dtype=torch.float32))
        self.pack()

    def forward(self, X, out=None, tcgen05=True):
        """X: BF16 [n][16] CUDA tensor -> FP32 [n][8] (columns 0..3 used).  tcgen05: the kernel on tcgen05 MMAs
        with TMEM accumulators (dphd_mlp_forward_tc), else the mma.sync kernel (dphd_mlp_forward)."""
        n = X.shape[0]
        if out is None:
            out = torch.empty(n, N_OUT, dtype=torch.float32, device=self.device)
        if tcgen05:
            if self._err is None:
                self._err = torch.zeros(1, dtype=torch.int32, device=self.device)
            core.Deformable._check(self._L.dphd_mlp_forward_tc(_p(self.master), _p(self.packed), _p(X), int(n),
                                                               _p(out), _p(self._err), self._stream()))
        else:
            core.Deformable._check(self._L.dphd_mlp_forward(_p(self.master), _p(self.packed), _p(X), int(n),
                                                            _p(out), self._stream()))
        return out

    def check_tensor_core_waits(self):
        """Raises if a tcgen05 inference kernel gave up a completion wait since the last check (synchronises)."""
        if self._err is not None and int(self._err.item()) != 0:
            self._err.zero_()
            raise RuntimeError("warm-start MLP: a tensor-core completion wait timed out")

    def _partials(self, n):
        blocks = (n + self.rows_per_block - 1) // self.rows_per_block
        need = blocks * self.part_per_block
        if self._part is None or self._part.numel() < need:
            self._part = torch.empty(need, dtype=torch.float32, device=self.device)
        return self._part

    def gradient(self, X, Y):
        """(mean loss, gradient) on rows X/Y without changing the weights or the optimiser state."""
        n = X.shape[0]
        grad = torch.zeros_like(self.master)
        core.Deformable._check(self._L.dphd_mlp_train_step(
            _p(self.master), _p(self.packed), _p(X), _p(Y), int(n), _p(self._partials(n)), 0.0, 0.9, 0.999, 1e-8,
            0.0, 1, _p(self.m), _p(self.v), _p(grad), _p(self.loss_buf), self._stream()))
        return self.loss_buf / n, grad

    def train_step(self, X, Y, lr, betas=(0.9, 0.999), eps=1e-8, weight_decay=1e-4, grad=None):
        """One AdamW step on the rows X (BF16 [n][16]), Y (FP32 [n][4]); returns the mean loss (device tensor,
        before the update)."""
        n = X.shape[0]
        self.step_count += 1
        core.Deformable._check(self._L.dphd_mlp_train_step(
            _p(self.master), _p(self.packed), _p(X), _p(Y), int(n), _p(self._partials(n)), float(lr),
            float(betas[0]), float(betas[1]), float(eps), float(weight_decay), int(self.step_count), _p(self.m),
            _p(self.v), _p(grad), _p(self.loss_buf), self._stream()))
        return self.loss_buf / n


class WarmStartStepper:
    """Forward steps of one deformable whose PD loops start from the network's prediction.

    `mlp=None` gives the non-learned extrapolation q_init = q_tilde + (q - q_tilde_prev) (the previous step's
    correction carried over), an ablation of the learned start."""

    def __init__(self, deformable, mlp, method, dt, options):
        self.d, self.mlp, self.method, self.dt, self.options = deformable, mlp, method, float(dt), dict(options)
        self.prev_base = None
        self.q_prev = None
        self._bufs = None

    def reset(self):
        self.prev_base = None
        self.q_prev = None

    def _alloc(self, like):
        n3 = like.numel()
        dev = like.device
        self._bufs = {
            "X": torch.empty(n3 // 3, N_IN, dtype=torch.bfloat16, device=dev),
            "base": [torch.empty(n3, dtype=torch.float64, device=dev) for _ in range(2)],
            "out": torch.zeros(n3 // 3, N_OUT, dtype=torch.float32, device=dev),
            "q_init": torch.empty(n3, dtype=torch.float64, device=dev),
            "q_prev": torch.empty(n3, dtype=torch.float64, device=dev),
            "which": 0,
        }

    def predict(self, q, v, f_ext, stream=0):
        """Features, network and q_init for one step (returns q_init and the step's q_tilde)."""
        if self._bufs is None or self._bufs["q_init"].numel() != q.numel():
            self._alloc(q)
        b = self._bufs
        base = b["base"][b["which"]]
        q_prev = self.q_prev if self.q_prev is not None else q
        self.d.warmstart_features(self.dt, q, q_prev, v, f_ext, self.prev_base, b["X"], base, stream=stream)
        if self.mlp is not None:
            self.mlp.forward(b["X"], out=b["out"])
        elif self.prev_base is not None:
            # extrapolation ablation: out = (q - q_tilde_prev)/dx is feature columns 6..8
            b["out"][:, :3] = b["X"][:, 6:9].float()
        self.d.warmstart_apply(self.dt, base, b["out"], b["q_init"], stream=stream)
        return b["q_init"], base

    def step(self, q, v, f_ext, q_next, v_next, stream=0):
        q_init, base = self.predict(q, v, f_ext, stream)
        self.d.forward_device_init(self.method, q, v, f_ext, self.dt, self.options, q_init, q_next, v_next,
                                   stream=stream)
        self.prev_base = base
        self._bufs["which"] ^= 1
        self._bufs["q_prev"].copy_(q)
        self.q_prev = self._bufs["q_prev"]


def generate_dataset(make_scene, seeds, steps, device, options=None, method="pd_eigen_alg_phd", stream=0,
                     drop_unconverged=True):
    """Rollouts of the plain solver (PD loop from q) on each seeded scene; per step and node the features and the
    targets (q_next - q_tilde)/dx and the frame's contact multiplier (scaled, 0 off the contact set).  Returns X
    (BF16 [N][16]) and Y (FP32 [N][4]) on `device`.  Frames whose PD loop stopped at max_pd_iter are left out
    (drop_unconverged): their iterates are no solution to learn."""
    Xs, Ys = [], []
    generate_dataset.dropped_frames = 0
    for seed in seeds:
        sc = make_scene(int(seed))
        d = core.from_scene(sc)
        opts = dict(options or sc.options)
        q = torch.as_tensor(sc.q0, device=device).clone()
        v = torch.as_tensor(sc.v0, device=device).clone()
        f = torch.as_tensor(sc.f_ext, device=device).clone()
        n3 = q.numel()
        qn, vn = torch.empty_like(q), torch.empty_like(q)
        # one step to put the factor on the device (features need it)
        d.reset_warm_start()
        d.forward_device(method, q, v, f, sc.dt, opts, qn, vn, stream=stream)
        q_prev, prev_base = q.clone(), None
        q, v = qn.clone(), vn.clone()
        bases = [torch.empty(n3, dtype=torch.float64, device=device) for _ in range(2)]
        for t in range(steps):
            X = torch.empty(n3 // 3, N_IN, dtype=torch.bfloat16, device=device)
            base = bases[t % 2]
            d.warmstart_features(sc.dt, q, q_prev, v, f, prev_base, X, base, stream=stream)
            d.forward_device(method, q, v, f, sc.dt, opts, qn, vn, stream=stream)
            Y = torch.empty(n3 // 3, N_USED, dtype=torch.float32, device=device)
            d.warmstart_target(sc.dt, qn, base, Y, stream=stream)
            if drop_unconverged and not d.frame_stats()[1][-1]:
                generate_dataset.dropped_frames += 1
            else:
                Xs.append(X)
                Ys.append(Y)
            q_prev, prev_base = q, base
            q, v = qn.clone(), vn.clone()
        del d
    return torch.cat(Xs), torch.cat(Ys)


def fit(mlp: WarmStartMLP, X, Y, steps=3000, batch=65536, lr=2e-3, weight_decay=1e-5, seed=0, log_every=0):
    """AdamW with cosine decay on random mini-batches; returns the per-step mean losses (host floats)."""
    N = X.shape[0]
    g = torch.Generator(device=X.device).manual_seed(int(seed))
    losses = []
    batch = min(batch, N)
    for it in range(steps):
        idx = torch.randint(0, N, (batch,), device=X.device, generator=g)
        lr_t = lr * 0.5 * (1 + math.cos(math.pi * it / max(steps, 1)))
        loss = mlp.train_step(X[idx].contiguous(), Y[idx].contiguous(), lr_t, weight_decay=weight_decay)
        if log_every and (it % log_every == 0 or it == steps - 1):
            losses.append((it, float(loss)))
    return losses


def evaluate(make_scene, seeds, steps, mlp, device, options=None, method="pd_eigen_alg_phd", stream=0,
             modes=("plain", "learned")):
    """Iterations per step and device time per step of each start on each seed, at the same dual gate.
    Modes: "plain" (PD loop from q, the reference's start), "extrapolated" (mlp-free ablation), "learned"."""
    res = {m: {"iters": [], "ms": [], "q_final": []} for m in modes}
    for seed in seeds:
        sc = make_scene(int(seed))
        d = core.from_scene(sc)
        opts = dict(options or sc.options)
        for mode in modes:
            q = torch.as_tensor(sc.q0, device=device).clone()
            v = torch.as_tensor(sc.v0, device=device).clone()
            f = torch.as_tensor(sc.f_ext, device=device).clone()
            qn, vn = torch.empty_like(q), torch.empty_like(q)
            d.reset_warm_start()
            st = None if mode == "plain" else WarmStartStepper(d, mlp if mode == "learned" else None, method,
                                                                sc.dt, opts)
            # warm-up step (factor upload, graphs)
            d.forward_device(method, q, v, f, sc.dt, opts, qn, vn, stream=stream)
            d.reset_frame_stats()
            d.reset_warm_start()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                if st is None:
                    d.forward_device(method, q, v, f, sc.dt, opts, qn, vn, stream=stream)
                else:
                    st.step(q, v, f, qn, vn, stream=stream)
                q, v = qn.clone(), vn.clone()
            e1.record()
            torch.cuda.synchronize()
            it, _cv = d.frame_stats()
            res[mode]["iters"].append(float(np.mean(it)))
            res[mode]["ms"].append(e0.elapsed_time(e1) / steps)
            res[mode]["q_final"].append(q.cpu().numpy())
        del d
    return res
