#!/usr/bin/env python
"""Benchmark: simulation steps/s of the projective-dynamics step + its adjoint on B200.

One bench "step" is one forward PD time step (run to the dual gate) plus the adjoint of that step
(backbone solve to the same tolerance, routing and per-element parameter gradients).  The
workload is the heterogeneous Neo-Hookean tet block (32x16x16 cells split into 5 tets: 40,960 tets,
9,537 nodes, per-element (mu_e, lambda_e) from a seeded two-phase blob field, nu 0.45, dt 5e-3).
Inputs are seeded synthetic meshes (no datasets).

Headline (`value`): the learned-warm-start step: FP32 bulk + FP64 refinement, every PD loop started from
the per-node MLP's prediction, every adjoint solve started from the previous (later) step's adjoint.  The
network is trained before timing, on the GPU by the library's own kernels, on plain-solver rollouts of
held-out material seeds (1..8; the timed scene is seed 0); its set-up time is reported, not timed.
`plain_fp64_gpu` is the same step in FP64 with the reference's starts (q for the PD loop, 0 for the adjoint),
both stopped by the same 1e-6 dual gate.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision f64|mixed]

value: K steps with inputs resident in HBM (device-pointer C-ABI entry points), CUDA events on the
library stream, L2 flushed (256 MB write) between steps outside the timed windows.
e2e: the same K steps through the host-buffer C-ABI calls (PyForward / PyBackward), host<->device copies
inside the timed region.
Multi-GPU: independent replicas (the path does not shard; no collective on the data path); value is the
sum of replica throughputs computed from the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "sim steps/s fwd+adjoint, learned-warmstart FP32 vs plain FP64 GPU @1e-6 res"
WORKLOAD = "nh_tet_block_32x16x16_5tet_heterogeneous"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _clock_worker(pci, index, period, stop, ready, out):
    """Clock sampler process: NVML read-only queries of one GPU until `stop` is set."""
    rows = []
    try:
        import pynvml as nv
        nv.nvmlInit()
        try:
            h = nv.nvmlDeviceGetHandleByPciBusId(pci.encode()) if pci else nv.nvmlDeviceGetHandleByIndex(index)
        except Exception:
            h = nv.nvmlDeviceGetHandleByIndex(index)
        names = [("hw_slowdown", nv.nvmlClocksEventReasonHwSlowdown),
                 ("hw_thermal_slowdown", nv.nvmlClocksEventReasonHwThermalSlowdown),
                 ("sw_thermal_slowdown", nv.nvmlClocksEventReasonSwThermalSlowdown),
                 ("sw_power_cap", nv.nvmlClocksEventReasonSwPowerCap)]
        first = True
        while True:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            rows.append((sm, mx, [n for n, bit in names if r & bit]))
            if first:
                ready.set()
                first = False
            if stop.wait(period):
                break
    except Exception:
        ready.set()
    out.put(rows)


class ClockSampler:
    """Samples SM clocks and throttle reasons of this rank's GPU every 50 ms while the timed region runs, from a
    separate process (NVML, read-only).  A sampler thread in this process would contend for the interpreter
    lock with the thread that issues the library calls; an nvidia-smi subprocess per sample would cost tens of
    milliseconds each."""

    def __init__(self, local_rank=0, period=0.05):
        self.local_rank = local_rank
        self.period = period
        self.rows = []
        self._p = None

    def __enter__(self):
        import multiprocessing as mp
        pci = ""
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.local_rank)
            pci = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
        except Exception:
            pass
        ctx = mp.get_context("spawn")
        self._stop, ready, self._q = ctx.Event(), ctx.Event(), ctx.Queue()
        self._p = ctx.Process(target=_clock_worker,
                              args=(pci, self.local_rank, self.period, self._stop, ready, self._q), daemon=True)
        self._p.start()
        ready.wait(30)
        return self

    def __exit__(self, *a):
        if self._p is None:
            return
        self._stop.set()
        try:
            self.rows = self._q.get(timeout=30)
        except Exception:
            self.rows = []
        self._p.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [r[0] for r in self.rows]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted({n for r in self.rows for n in r[2]}), "samples": len(self.rows),
                "source": "NVML, 50 ms period, separate process"}


SCENE = "nh_tet_block"


def build_scene(name=None):
    """The bench workload, or (for kernel-only profiling) the 24^3 hex block without contact, whose S is
    larger than L2."""
    from diffphd_b200 import scenes
    name = name or SCENE
    if name == "nh_tet_block":
        return scenes.nh_tet_block()
    if name == "hex24":
        sc = scenes.contact_drop()
        sc.plane = None
        return sc
    raise SystemExit(f"unknown scene {name}")


def run_contact_drop(args):
    """Secondary measurement on the contact-rich drop (24^3 hex block, E 5e5, nu 0.4, seeded rotation, dropped
    onto z = 0, Coulomb mu 0.5, every node a candidate): W untimed FP64 steps bring the block into contact,
    then K forward steps + their adjoints are timed in FP64 (reference starts) and in mixed precision with the
    adjoint warm start.  Not the headline workload."""
    import torch
    from diffphd_b200 import core, scenes
    dev = torch.device("cuda", 0)
    sc = scenes.contact_drop()
    out = {"metric": "sim steps/s fwd+adjoint, contact-rich drop (secondary)", "unit": "steps/s",
           "config": {"workload": "contact_drop_hex_24x24x24_mu0.5", "nodes": sc.n, "elements": sc.m,
                      "candidates": int(len(sc.plane[1])), "dt": sc.dt, "pre_contact_steps": args.warmup}}
    for name, prec, warm in (("fp64", "f64", False), ("mixed_adjoint_warm", "mixed", True)):
        d = core.from_scene(sc)
        opts = options(sc, prec, warm=warm)
        T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev).contiguous()
        f = T(sc.f_ext)
        q, v = T(sc.q0), T(sc.v0)
        qn, vn = torch.empty_like(q), torch.empty_like(q)
        o64 = options(sc, "f64")
        for _ in range(args.warmup):  # free fall into contact
            d.forward_device("pd_eigen_alg_phd", q, v, f, sc.dt, o64, qn, vn)
            q, v = qn.clone(), vn.clone()
        d.reset_frame_stats()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        qs, vs = [q], [v]
        e0.record()
        for _ in range(args.steps):
            qn, vn = torch.empty_like(q), torch.empty_like(q)
            d.forward_device("pd_eigen_alg_phd", qs[-1], vs[-1], f, sc.dt, opts, qn, vn)
            qs.append(qn)
            vs.append(vn)
        g, gv = T(sc.extra.get("loss_r", np.ones(sc.dofs))), torch.zeros_like(q)
        bw = []
        for i in reversed(range(args.steps)):
            dq, dv, df = torch.empty_like(g), torch.empty_like(g), torch.empty_like(g)
            d.backward_device("pd_eigen_alg_phd", qs[i + 1], g, gv, sc.dt, opts, dq, dv, df)
            bw.append(d._L.dphd_last_backward_iters(d._h))
            g, gv = dq, dv
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        it, cv = d.frame_stats()
        act = len(d.contact_lambda().nonzero())
        out[name] = {"value": args.steps / t, "ms_per_step": t / args.steps * 1e3,
                     "pd_iters_per_step": float(np.mean(it)), "adjoint_iters_per_step": float(np.mean(bw)),
                     "converged_frac": float(np.mean(cv)), "active_contacts_last": int(act)}
    out["speedup_mixed"] = out["mixed_adjoint_warm"]["value"] / out["fp64"]["value"]
    print(json.dumps(out), flush=True)


def run_ainv_only(args):
    """Kernel-only mode for profiling: builds the scene's factor, then applies the S^T S pair `reps` times."""
    import numpy as np
    from diffphd_b200 import core
    sc = build_scene(args.scene)
    d = core.from_scene(sc)
    fp32 = args.precision == "mixed"
    d.debug_ainv(np.ones(sc.dofs), sc.dt, fp32=fp32)
    ms = d.time_ainv(sc.dt, reps=args.ainv_reps, fp32=fp32, flush_l2=False)
    print(json.dumps({"scene": args.scene, "precision": args.precision, "ms_per_apply": ms, "nnz_S": d.s_nnz(),
                      "stored_values": d.s_padded_values()}))


HOST_LOOP = False  # --host-loop: iteration loops replayed from the host (profilers see each kernel launch)


def options(sc, precision, warm=False):
    o = dict(sc.options)
    o["thread_ct"] = os.cpu_count() or 8
    if HOST_LOOP:
        o["graph_while"] = 0
    o["alg_phd_bwd_solver"] = 1   # conjugate-gradient adjoint, stopped by the reference's 1e-6 step rule
    if precision == "mixed":
        o["fp32_bulk"] = 1
    if warm:
        o["alg_phd_bwd_warm_start"] = 3  # quadratic extrapolation of the last three adjoints of the sweep
    return o


def max_over_ranks(values, world, dev):
    """Each value's maximum over the ranks of the process group (the slowest replica sets the job's time);
    the values themselves when running alone."""
    if world <= 1:
        return [float(x) for x in values]
    import torch
    t = torch.tensor([float(x) for x in values], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def train_warm_start(dev, args):
    """Trains the warm-start MLP on plain-solver rollouts of held-out material seeds (not the timed seed 0)."""
    import torch
    from diffphd_b200 import scenes
    from diffphd_b200.warmstart import WarmStartMLP, fit, generate_dataset
    seeds = list(range(1, 1 + args.ws_seeds))
    sc0 = build_scene()
    t0 = time.perf_counter()
    X, Y = generate_dataset(lambda s: scenes.nh_tet_block(seed=s), seeds, args.ws_steps, dev,
                            options=options(sc0, "mixed"))
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    mlp = WarmStartMLP(dev, seed=0)
    hist = fit(mlp, X, Y, steps=args.ws_fit_steps, batch=65536, lr=2e-3, log_every=max(1, args.ws_fit_steps - 1))
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    info = {"train_seeds": f"{seeds[0]}..{seeds[-1]}", "rollout_steps_per_seed": args.ws_steps, "rows": int(X.shape[0]),
            "data_gen_s": round(t1 - t0, 2), "fit_s": round(t2 - t1, 2), "fit_steps": args.ws_fit_steps,
            "batch": 65536, "loss_first_last": [h[1] for h in hist]}
    del X, Y
    return mlp, info


def cpu_baseline(sc, opts, steps=1):
    """Times the oracle (CPU restatement of the reference path, OpenMP on all host cores) on a bounded
    sample: `steps` forward steps and their adjoints from the scene's rest state."""
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    o = oracle.OracleDeformable.from_scene(sc)
    copts = dict(opts)
    copts.pop("fp32_bulk", None)
    copts.pop("alg_phd_bwd_solver", None)
    copts.pop("alg_phd_bwd_warm_start", None)
    copts["thread_ct"] = cores
    t_setup = time.perf_counter()
    o.ainv(np.zeros(sc.dofs), sc.dt)  # factorization, reported separately (not in the sample)
    t_setup = time.perf_counter() - t_setup
    q, v = sc.q0.copy(), sc.v0.copy()
    qs, vs = [q], [v]
    t0 = time.perf_counter()
    for _ in range(steps):
        q, v, _ = o.forward(q, v, sc.f_ext, sc.dt, copts)
        qs.append(q)
        vs.append(v)
    g = sc.extra["loss_r"].copy()
    gv = np.zeros(sc.dofs)
    for i in reversed(range(steps)):
        out = o.backward(qs[i], vs[i], sc.f_ext, sc.dt, qs[i + 1], g, gv, copts)
        g, gv = out["dl_dq"], out["dl_dv"]
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": "steps/s", "cores": cores, "kind": "port",
            "sample": f"{steps} forward step(s) + adjoint(s) of {WORKLOAD} from rest, oracle FP64, "
                      f"factorization {t_setup:.2f}s excluded"}


def run_ours(args, rank, world, local_rank):
    import torch
    from diffphd_b200 import core
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    sc = build_scene()
    d = core.from_scene(sc)
    learned = args.precision == "mixed" and not args.no_warm_start
    mlp, ws_info = (train_warm_start(dev, args) if learned else (None, None))
    line = _measure(args, rank, world, local_rank, args.precision, True, sc, d, mlp, warm=learned)
    if args.precision == "mixed" and not args.no_fp64_compare:
        ref = _measure(args, rank, world, local_rank, "f64", False, sc, d, None, warm=False)
        abl = _measure(args, rank, world, local_rank, "mixed", False, sc, d, None, warm=False) if learned else None
        if line is not None and ref is not None:
            line["plain_fp64_gpu"] = {"value": ref["value"], "unit": "steps/s", "ms_per_step": ref["ms_per_step"],
                                      "pd_iters_per_step": ref["pd_iters_per_step"],
                                      "adjoint_iters_per_step": ref["adjoint_iters_per_step"],
                                      "speedup_of_headline": line["value"] / ref["value"]}
            if abl is not None:
                line["mixed_without_warm_starts"] = {
                    "value": abl["value"], "unit": "steps/s", "ms_per_step": abl["ms_per_step"],
                    "pd_iters_per_step": abl["pd_iters_per_step"],
                    "adjoint_iters_per_step": abl["adjoint_iters_per_step"]}
    if line is not None and ws_info is not None:
        line["warm_start_network"] = ws_info
    if line is not None and not args.no_cpu_baseline:
        # last: the oracle's OpenMP threads would otherwise compete with the host side of the GPU timings
        line["cpu_baseline"] = cpu_baseline(sc, options(sc, "f64"), steps=1)
    return line


def _measure(args, rank, world, local_rank, precision, full, sc, d, mlp, warm):
    import torch
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    opts = options(sc, precision, warm=warm)
    d.set_warm_start_network(mlp)
    n3 = sc.dofs
    method = "pd_eigen_alg_phd"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    T = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), device=dev).contiguous()
    f_ext = T(sc.f_ext)
    g_final = T(sc.extra["loss_r"])
    zeros = torch.zeros(n3, dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream

    def roll(q0, v0, k):
        qs, vs = [q0], [v0]
        for _ in range(k):
            qn, vn = torch.empty_like(q0), torch.empty_like(q0)
            d.forward_device(method, qs[-1], vs[-1], f_ext, sc.dt, opts, qn, vn, stream=sh)
            qs.append(qn)
            vs.append(vn)
        return qs, vs

    # warm-up: W steps forward + adjoint (builds S, captures the iteration graphs)
    d.reset_warm_start()
    with torch.cuda.stream(stream):
        qs, vs = roll(T(sc.q0), T(sc.v0), args.warmup)
        gq, gv = g_final.clone(), zeros.clone()
        for i in reversed(range(args.warmup)):
            dq, dv, df = torch.empty_like(gq), torch.empty_like(gq), torch.empty_like(gq)
            d.backward_device(method, qs[i + 1], gq, gv, sc.dt, opts, dq, dv, df, stream=sh)
            gq, gv = dq, dv
    stream.synchronize()
    q_start, v_start = qs[-1], vs[-1]
    d.reset_frame_stats()

    # timed region 1 (value): device-resident inputs; the warm starts carry state only within this rollout
    d.reset_warm_start()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = d.kernel_launches()
    ev = []
    bwd_iters = []
    with ClockSampler(local_rank) as clk, torch.cuda.stream(stream):
        torch.cuda.nvtx.range_push("timed_value")  # lets a profiler restrict itself to the timed steps
        q, v = q_start, v_start
        qs, vs = [q], [v]
        # every output is allocated before the timed region: an allocator call inside an event window would be
        # timed as device time
        q_out = [(torch.empty_like(q), torch.empty_like(q)) for _ in range(args.steps)]
        g_out = [(torch.empty_like(q), torch.empty_like(q), torch.empty_like(q)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.random_(0, 255)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            qn, vn = q_out[k]
            e0.record(stream)
            d.forward_device(method, qs[-1], vs[-1], f_ext, sc.dt, opts, qn, vn, stream=sh)
            e1.record(stream)
            ev.append((e0, e1))
            qs.append(qn)
            vs.append(vn)
        gq, gv = g_final.clone(), zeros.clone()
        dpar = torch.empty(max(1, d.NumOfPdParams()), dtype=torch.float64, device=dev)
        for i in reversed(range(args.steps)):
            flush.random_(0, 255)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            dq, dv, df = g_out[i]
            e0.record(stream)
            d.backward_device(method, qs[i + 1], gq, gv, sc.dt, opts, dq, dv, df, dl_dparams=dpar, stream=sh)
            e1.record(stream)
            ev.append((e0, e1))
            bwd_iters.append(d._L.dphd_last_backward_iters(d._h))
            gq, gv = dq, dv
        stream.synchronize()
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches = d.kernel_launches() - launches0
    t_dev = sum(a.elapsed_time(b) for a, b in ev) / 1e3
    fwd_iters, conv = d.frame_stats()

    if not full:
        (t_dev,) = max_over_ranks([t_dev], world, dev)
        if rank != 0:
            return None
        return {"value": args.steps * world / t_dev, "ms_per_step": t_dev / args.steps * 1e3,
                "pd_iters_per_step": float(np.mean(fwd_iters)) if len(fwd_iters) else None,
                "adjoint_iters_per_step": float(np.mean(bwd_iters)) if bwd_iters else None}

    # timed region 2 (e2e): host buffers through the C ABI (PyForward / PyBackward; the attached network and
    # the adjoint warm start act behind the same calls)
    qh, vh = q_start.cpu().numpy(), v_start.cpu().numpy()
    d.reset_warm_start()
    fh = np.asarray(sc.f_ext)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t_e2e = 0.0
    qs_h, vs_h = [qh], [vh]
    for _ in range(args.steps):
        flush.random_(0, 255)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        qn, vn = np.zeros(n3), np.zeros(n3)
        d.PyForward(method, qs_h[-1], vs_h[-1], [], fh, sc.dt, opts, qn, vn, [])
        t_e2e += time.perf_counter() - t0
        qs_h.append(qn)
        vs_h.append(vn)
    gq_h, gv_h = np.asarray(sc.extra["loss_r"]), np.zeros(n3)
    for i in reversed(range(args.steps)):
        flush.random_(0, 255)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = d.backward(method, qs_h[i], vs_h[i], [], fh, sc.dt, qs_h[i + 1], vs_h[i + 1], [], gq_h, gv_h, opts)
        t_e2e += time.perf_counter() - t0
        gq_h, gv_h = out["dl_dq"], out["dl_dv"]
    if world > 1:
        torch.distributed.barrier()

    t_dev, t_e2e = max_over_ranks([t_dev, t_e2e], world, dev)
    if rank != 0:
        return None

    # roofline of the dominant kernel pair (S v, S^T y): algorithmic bytes per A^-1 apply (3 RHS)
    fp32 = precision == "mixed"
    nnz = d.s_nnz()
    n = sc.n
    alg = 2 * nnz * (8 if fp32 else 12) + 4 * 3 * n * (4 if fp32 else 8)
    raw = 2 * d.s_padded_values() * (4 if fp32 else 8) + 4 * 3 * n * (4 if fp32 else 8)
    ms = d.time_ainv(sc.dt, reps=30, fp32=fp32, flush_l2=True)
    peak, peak_kind = _peaks()
    achieved = alg / (ms * 1e-3) / 1e9
    traffic = None
    tp = ROOT / "profiles" / "sts_pair_traffic.json"
    if tp.exists():
        tj = json.loads(tp.read_text())
        traffic = tj.get("f32" if fp32 else "f64")
    steps_total = args.steps * world
    h2d = 3 * n3 * 8 + 3 * n3 * 8      # forward: q, v, f_ext; adjoint: q_next, dl_dq_next, dl_dv_next
    d2h = 2 * n3 * 8 + 3 * n3 * 8 + 8 * (d.NumOfPdParams() + d.NumOfPdElementEnergies() + 3)
    line = {
        "metric": METRIC,
        "value": steps_total / t_dev,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_dev / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64" if fp32 else "f64",
        "data": "synthetic (seeded two-phase blob material field, rest-state start)",
        "config": {"workload": WORKLOAD, "nodes": n, "elements": sc.m, "dt": sc.dt,
                   "precision": "fp32 bulk (projection, S/S^T) + fp64 gate/AA" if fp32 else "plain fp64",
                   "pd_start": "learned warm start (per-node MLP, BF16 tensor cores)" if mlp is not None
                   else "q (reference)",
                   "adjoint_start": "3 (mu_1 - mu_2) + mu_3 (last three adjoints of the sweep)" if warm else "0 (reference)",
                   "rel_tol": opts["rel_tol"], "abs_tol": opts["abs_tol"], "aa_window": opts["aa_window"],
                   "max_pd_iter": opts["max_pd_iter"], "step": "forward PD step + adjoint step",
                   "adjoint_solver": "PCG on (A - K_pd) preconditioned by S^T S, FP64 residual",
                   "l2": "flushed (256 MB write) between steps, outside the timed windows",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "roofline": {"bound": "hbm", "kernel": "S v + S^T y pair (3 RHS)", "achieved": achieved, "peak": peak,
                     "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "ms_per_apply": ms, "algorithmic_bytes": alg, "raw_bytes_streamed": raw, "nnz_S": nnz},
        "e2e": {"value": steps_total / t_e2e, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
        "pd_iters_per_step": float(np.mean(fwd_iters)) if len(fwd_iters) else None,
        "adjoint_iters_per_step": float(np.mean(bwd_iters)) if bwd_iters else None,
        "forward_converged_frac": float(np.mean(conv)) if len(conv) else None,
        # device time of each timed call (forward steps, then the adjoints in reverse order), for the spread
        "call_ms": [round(a.elapsed_time(b), 3) for a, b in ev],
    }
    return line


def run_reference(args, rank, world):
    if rank != 0:
        return None
    sc = build_scene()
    opts = options(sc, "f64")
    vals = []
    for _ in range(args.warmup):
        pass  # the CPU port has no warm-up state beyond its factorization (done inside cpu_baseline)
    for _ in range(max(1, min(args.steps, 2))):
        vals.append(cpu_baseline(sc, opts, steps=1))
    v = float(np.mean([x["value"] for x in vals]))
    cb = dict(vals[0])
    cb["value"] = v
    return {"metric": METRIC, "impl": "reference", "value": v, "unit": "steps/s", "n_gpus": world,
            "steps": len(vals), "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nodes": sc.n, "elements": sc.m, "dt": sc.dt,
                       "note": "reference has no buildable GPU path here; its CPU algorithm is timed via the "
                               "oracle port (OpenMP, all host cores), bounded sample per step"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["f64", "mixed"])
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--scene", default="nh_tet_block", choices=["nh_tet_block", "hex24"])
    ap.add_argument("--ainv-reps", type=int, default=0,
                    help="profiling mode: only apply the S^T S pair this many times on --scene")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--contact-drop", action="store_true",
                    help="secondary measurement: the contact-rich 24^3 drop (--warmup = untimed free-fall steps)")
    ap.add_argument("--no-warm-start", action="store_true", help="headline without the learned / adjoint starts")
    ap.add_argument("--host-loop", action="store_true",
                    help="profiling: replay each iteration graph from the host instead of one device-side WHILE "
                         "graph per solve (same kernels; ncu does not profile kernels inside conditional nodes)")
    ap.add_argument("--ws-seeds", type=int, default=12, help="material seeds of the warm-start training rollouts")
    ap.add_argument("--ws-steps", type=int, default=60, help="rollout steps per training seed")
    ap.add_argument("--ws-fit-steps", type=int, default=4000, help="AdamW steps of warm-start training")
    args = ap.parse_args()
    global HOST_LOOP
    HOST_LOOP = args.host_loop
    if args.warmup < 3:
        args.warmup = 3
    if args.ainv_reps > 0:
        run_ainv_only(args)
        return
    if args.contact_drop:
        run_contact_drop(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference" and rank != 0:
        return  # the reference arm runs on rank 0 only
    if world > 1 and args.impl == "ours":
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world)
        else:
            line = run_ours(args, rank, world, local_rank)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1 and args.impl == "ours":
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
