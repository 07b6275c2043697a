#!/usr/bin/env python
"""Benchmark of swfwi's batched FWI gradient on B200.

One step = one batched FWI gradient over all 96 shots of the 301 x 921 grid
(dx 10 m, dt 1 ms, nt 4000, 15 Hz Ricker, 30-point sponge, seeded uneven
receiver spreads of 200-921 points): forward modelling with boundary-strip
save, direct-arrival mute, residual and FP64 objective, time derivative,
back-propagation of the source field with adjoint receiver propagation and
imaging, gradient scale/mask and the sum over shots.  Inputs are resident in
HBM when the timed region starts (the velocity, the wavelet and all observed
shots, 0.6 GB).

Arithmetic: FP32 with FMA by default (seismograms within 1e-5, gradients
within 1e-4 relative L2 of the reference, the tests' bounds); --arith ref
reproduces the reference's float/double rounding bit for bit.  --fuse on
runs the backward time loop fused (source subtraction and imaging in the
source back-step, residual injection in the receiver step).

value: stencil point-updates executed per second over the timed steps
(Gpts/s), device-timed with CUDA events, max over ranks.  e2e: the same
gradient through the C ABI from pinned host buffers, host-device copies
inside the timed region.  --impl reference: the reference's own CPU code
(oracle/_ref, OpenMP over all host cores) on a bounded sample of the same
workload.

Multi-GPU: replicas only (the workload runs on one GPU; N ranks run N
independent copies, value = all ranks' point-updates / max time).

Other modes: --mode tune (the autotuner's table), --mode kernel (a short
96-shot batched forward, the small case for ncu), --mode learned (FWI
wall-clock to equal model error, learned preconditioner vs plain, on seeded
gradient + anomaly models of 240 x 80 with held-out test models), --mode
network (the preconditioner's kernels alone).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FD Gpts/s (% HBM roofline); FWI wall-clock to equal model L2, learned vs plain"
CONFIG = "batched"
CPU_SAMPLE_NT = 1500
CPU_SAMPLE_NT_ASBUILT = 600
TIMING_PERIOD = 16


def max_over_ranks(x: float, dist=None, device="cuda") -> float:
    """The largest value of a per-rank scalar over all ranks (a job's time
    is its slowest rank's); dist None: one rank."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(updates_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job Gpts/s of N replicas: every rank's point-updates over the
    slowest rank's time."""
    return updates_per_rank * world / seconds_max / 1e9


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes per point-update of each stencil kernel on the 96-shot
# workload's launch (993 x 343 padded, 31,172,256 point-updates), from one
# ncu capture: (dram__bytes_read.sum + dram__bytes_write.sum) / point-updates.
# Kernel 1: 288.79 MB + 88.67 MB (profiles/fd_step_ws_96shots_993x343_fast.md);
# kernel 5 with its automatic task length (99 rows): 282.84 MB + 87.86 MB
# (profiles/fd_step_rq_96shots_993x343_fast.md; part of the writes is still
# in L2 when the launch ends); kernel 6 with its automatic task length (123
# rows): 279.60 MB + 87.87 MB (profiles/fd_step_rq2_96shots_993x343_fast.md).
STENCIL_TRAFFIC_B_PER_PT = {1: 12.11, 5: 11.89, 6: 11.79}


def traffic_per_point(kernel):
    return STENCIL_TRAFFIC_B_PER_PT.get(kernel)


def backward_steps(nt: int, dt: float) -> int:
    """Back-propagation steps calgradient performs (fwiframework.cpp:146-176):
    it runs from nt-1 down and stops after the first step with dt*it <= 0.3 s."""
    n = 0
    dt32 = np.float32(dt)
    for it in range(nt - 1, -1, -1):
        n += 1
        t = float(np.float32(dt32 * np.float32(it)))
        if not t > 0.3:
            break
    return n


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, fl in rows for i, v in enumerate(fl) if v.lower() == "active"})
        sm = sorted(r[0] for r in rows)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


def setup_workload(torch, arith, nt=0):
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    s = sv.config(CONFIG)
    if nt > 0:
        s = s.scaled(nt=nt)
    vtrue = sv.layered_model(s.nx, s.nz, seed=2024)
    vinit = sv.smooth(vtrue, 15.0).astype(np.float32)
    m = S.Damp4t10d.from_survey(s, arith=arith)
    ext = torch.from_numpy(m.expandDomain(vtrue)).cuda()
    exi_h = m.expandDomain(vinit)
    exi = torch.from_numpy(exi_h).cuda()
    wlt_h = S.ricker_wavelet(s.nt, s.fm, s.dt, 1.0)
    wlt = torch.from_numpy(wlt_h).cuda()
    ids = np.arange(s.ns, dtype=np.int32)
    nxpad, nzpad, ns, ngmax, nt = m.dims()
    dobs = torch.zeros((ns, nt, ngmax), dtype=torch.float32, device="cuda")
    m.bindVelocity(ext)
    m.forward_batch(wlt, dobs, ids)          # observed data: the true model
    m.bindVelocity(exi)
    torch.cuda.synchronize()
    return s, m, exi, exi_h, wlt, wlt_h, dobs, ids


def cpu_reference_sample(nt_sample=CPU_SAMPLE_NT, repeats=1, asbuilt=False):
    """The reference's gradient loop on one shot of the workload with the
    time axis cut to nt_sample steps, OpenMP over all host cores (asbuilt:
    the reference as its own build compiles it, pass 1 of the damped step
    serial).  Also returns what the GPU needs to recompute the same sample
    and the reference's gradient and objective to check it against."""
    import oracle
    from swfwi_b200 import survey as sv
    if not oracle.available():
        return None
    s = sv.config(CONFIG)
    off, gx, _ = s.spreads
    n0 = int(off[1] - off[0])
    ss = s.scaled(nt=nt_sample, ns=1, ng=n0, gxbeg=int(gx[0]), spreads=None)
    R = oracle.RefLib(asbuilt=asbuilt)
    M = R.model(ss)
    vtrue = sv.layered_model(s.nx, s.nz, seed=2024)
    vinit = sv.smooth(vtrue, 15.0).astype(np.float32)
    wlt = R.ricker(ss.nt, ss.fm, ss.dt)
    M.expand_domain(vtrue)
    dobs = M.fwi_forward(wlt, 0)[None]
    M.expand_domain(vinit)
    pts = (M.nxpad - 12) * (M.nzpad - 12)
    updates = pts * (2 * ss.nt + 2 * backward_steps(ss.nt, ss.dt))
    times = []
    grad = obj = None
    for _ in range(repeats):
        t0 = time.perf_counter()
        grad, obj = M.fwi_gradient(wlt, dobs)
        times.append(time.perf_counter() - t0)
    return {"seconds": min(times), "updates": updates, "cores": _cores(),
            "sample": f"one shot ({n0} receivers), nt={ss.nt}, full {M.nxpad}x{M.nzpad} padded grid, "
                      f"reference gradient loop (FwiForwardModeling, mute, residual, transVsrc, "
                      f"calgradient, scale/mask)" + (", as built (pass 1 serial)" if asbuilt else ""),
            "survey": ss, "vinit": vinit, "wlt": wlt, "dobs": dobs, "grad": grad, "obj": obj}


def parity_of_sample(torch, arith, tuning, info):
    """The product's gradient of the CPU-baseline sample (the same shot,
    velocity, wavelet and observed data) against the reference's gradient
    of it: relative L2 and objective difference."""
    import swfwi_b200 as S
    ss = info["survey"]
    m = S.Damp4t10d.from_survey(ss, arith=arith)
    m.set_tuning(**tuning)
    vel = torch.from_numpy(m.expandDomain(info["vinit"])).cuda()
    m.bindVelocity(vel)
    gr = torch.zeros(vel.shape, device="cuda")
    obj = m.gradient_batch(torch.from_numpy(np.ascontiguousarray(info["wlt"])).cuda(),
                           torch.from_numpy(np.ascontiguousarray(info["dobs"])).cuda(), [0], gr)
    g = gr.cpu().numpy().astype(np.float64)
    want = np.asarray(info["grad"], np.float64)
    e = float(np.linalg.norm(g - want) / np.linalg.norm(want))
    eo = float(abs(float(obj.sum()) - info["obj"]) / abs(info["obj"]))
    return {"case": "the CPU baseline's sample: " + info["sample"], "grad_rel_l2": e, "objective_rel": eo,
            "tolerance": {"grad_rel_l2": 1e-4, "objective_rel": 1e-4},
            "ok": bool(e < 1e-4 and eo < 1e-4)}


def run_reference(args):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    import oracle
    if not oracle.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference compiled "
                          "from its sources) is not built"}))
        return 0
    for _ in range(args.warmup):
        cpu_reference_sample(repeats=1)
    tot_t, tot_u, info = 0.0, 0, None
    for _ in range(args.steps):
        info = cpu_reference_sample(repeats=1)
        tot_t += info["seconds"]
        tot_u += info["updates"]
    v = tot_u / tot_t / 1e9
    line = {"metric": METRIC, "value": v, "unit": "Gpts/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_t / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "batched FWI gradient, 96 shots, 301x921 grid (993x337 padded), nt=4000, "
                                   "uneven spreads 200-921",
                       "sample": f"each step a bounded sample of that workload: {info['sample']}",
                       "arith": "reference float arithmetic (the reference's own CPU code, OpenMP)"},
            "cpu_baseline": {"value": v, "unit": "Gpts/s", "cores": info["cores"], "kind": "reference",
                             "sample": info["sample"]},
            "e2e": {"value": v, "unit": "Gpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_kernel_mode(args):
    """Short batched forward runs on the workload's grid and shots: the
    autotuner's table (--mode tune) or one run at the tuned shape
    (--mode kernel, the small case for profiling)."""
    import torch
    import swfwi_b200 as S
    from swfwi_b200 import autotune
    from swfwi_b200 import survey as sv
    arith = S.ARITH_REF if args.arith == "ref" else S.ARITH_FAST
    s = sv.config(CONFIG)
    vtrue = sv.layered_model(s.nx, s.nz, seed=2024)
    m0 = S.Damp4t10d.from_survey(s)
    ex = m0.expandDomain(vtrue)
    if args.mode == "tune":
        best, table = autotune.tune(s, ex, arith, nt_probe=args.nt, verbose=True)
        pts = (s.nxpad - 12) * (s.nzpad - 12) * s.ns
        for us, cfg in table[:5]:
            print(json.dumps({"us_per_launch": us, "gpts": pts / us / 1e3,
                              "gbs": pts * 12.04 / us / 1e3, **cfg}))
        return 0
    ss = s.scaled(nt=args.nt)
    m = S.Damp4t10d.from_survey(ss, arith=arith)
    m.set_tuning(**(json.loads(args.tuning) if args.tuning else autotune.DEFAULT))
    m.set_fusion(args.fuse == "on")
    vel = torch.from_numpy(ex).cuda()
    m.bindVelocity(vel)
    wlt = torch.from_numpy(S.ricker_wavelet(ss.nt, ss.fm, ss.dt)).cuda()
    ids = np.arange(ss.ns, dtype=np.int32)
    dcal = torch.zeros((ss.ns, ss.nt, m.getng()), device="cuda")
    m.forward_batch(wlt, dcal, ids)
    torch.cuda.synchronize()
    print(json.dumps({"mode": "kernel", "shots": ss.ns, "nt": ss.nt,
                      "checksum": float(dcal.abs().sum().item())}))
    return 0


# ---------------------------------------------------------------- the other workload configurations
def _timed(torch, fn):
    """Wall seconds of fn() between two device synchronisations."""
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = fn()
    torch.cuda.synchronize()
    return time.perf_counter() - t0, r


def _cpu_timed(fn):
    t0 = time.perf_counter()
    r = fn()
    return time.perf_counter() - t0, r


def record_fwi_iteration(torch, arith, tuning, cpu):
    """Plain FWI, one iteration: 20 shots of 151 x 461 (193 x 533 padded),
    nt 2000, dt 2 ms, 10 Hz: the batched gradient of all shots, the
    step-length search with its trial forwards, the velocity update
    (FwiFramework::epoch, fwiframework.cpp:269-356).  GPU seconds are the
    second epoch's (the first allocates).  The reference CPU seconds are
    extrapolated from its own per-shot units timed at full nt on the host
    cores: 20 x (one shot's gradient loop + trials x one shot's forward),
    trials = the trial objectives this run's search evaluated."""
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    s = sv.config("fwi")
    vt = sv.layered_model(s.nx, s.nz, seed=2024)
    vi = sv.smooth(vt, 15.0).astype(np.float32)
    m = S.Damp4t10d.from_survey(s, arith=arith)
    m.set_tuning(**tuning)
    ext, exi = m.expandDomain(vt), m.expandDomain(vi)
    wlt = S.ricker_wavelet(s.nt, s.fm, s.dt)
    vel = torch.from_numpy(ext).cuda()
    m.bindVelocity(vel)
    dobs = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
    m.forward_batch(torch.from_numpy(wlt).cuda(), dobs, np.arange(s.ns, dtype=np.int32))
    f = S.FwiFramework(m, exi, s.vmin, s.vmax, s.nita, s.maxdv, wlt, dobs.cpu().numpy())
    t_first, _ = _timed(torch, lambda: f.epoch(0))
    t_iter, _ = _timed(torch, lambda: f.epoch(1))
    trials = f.lastTrials()
    rec = {"workload": "plain FWI iteration: 20 shots, 151x461 (193x533 padded), nt 2000, dt 2 ms, 10 Hz, "
                       "gradient + step-length search + velocity update",
           "gpu_s": t_iter, "gpu_first_epoch_s": t_first, "trials": trials,
           "objective": f.getInitObj(), "objective_after": f.getUpdateObj()}
    if cpu:
        import oracle
        if oracle.available():
            R = oracle.RefLib()
            ss = s.scaled(ns=1, sxbeg=int(s.src_x()[s.ns // 2]))
            M = R.model(ss)
            M.expand_domain(vt)
            d1 = M.fwi_forward(wlt, 0)
            M.expand_domain(vi)
            tg, _ = _cpu_timed(lambda: M.fwi_gradient(wlt, d1[None]))
            tf, _ = _cpu_timed(lambda: M.fwi_forward(wlt, 0))
            cpu_s = s.ns * (tg + trials * tf)
            rec["cpu"] = {"s": cpu_s, "kind": "reference", "cores": _cores(),
                          "basis": f"extrapolated: 20 x (one shot's gradient loop {tg:.2f} s + {trials} x one "
                                   f"shot's forward {tf:.2f} s), each timed once at full nt"}
            rec["speedup_vs_cpu"] = cpu_s / t_iter
    return rec


def record_encoded(torch, arith, tuning, iters):
    """Encoded-source FWI: the 96 shots of 301 x 921 (nt 4000, dt 1 ms,
    15 Hz, common receiver line) as one supershot with +-1 codes re-drawn
    every iteration (EssFwiFramework::epoch, essfwiframework.cpp:191-239).
    `iters` iterations are timed (the 50-iteration run is their mean x 50).
    The gradient's error against the FP64 GPU run of the same scheme is
    stated for FP32, FP16 and BF16 boundary strips, on one supershot, and on
    the gradient's unmasked interior also for FP32, FP16 and BF16 checkpoint
    snapshots (every 64 steps), with one supershot gradient timed each way."""
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    s = sv.config("encoded")
    vt = sv.layered_model(s.nx, s.nz, seed=2024)
    vi = sv.smooth(vt, 15.0).astype(np.float32)
    m = S.Damp4t10d.from_survey(s, arith=arith)
    m.set_tuning(**tuning)
    ext, exi = m.expandDomain(vt), m.expandDomain(vi)
    wlt_h = S.ricker_wavelet(s.nt, s.fm, s.dt)
    wlt = torch.from_numpy(wlt_h).cuda()
    vel = torch.from_numpy(ext).cuda()
    m.bindVelocity(vel)
    dobs = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
    m.forward_batch(wlt, dobs, np.arange(s.ns, dtype=np.int32))
    velinit = torch.from_numpy(exi).cuda()
    m.bindVelocity(velinit)
    # the gradient of one supershot against FP64
    codes = torch.from_numpy(S.random_codes(1, s.ns)).cuda()
    encsrc = torch.empty((s.nt, s.ns), device="cuda")
    S.encode_source(encsrc, wlt, codes)
    encobs = torch.empty((s.nt, s.ng), device="cuda")
    S.encode_obs(encobs, dobs, codes)
    dcal = torch.zeros((s.nt, s.ng), device="cuda")
    m.EssForwardModeling(encsrc, dcal)
    vsrc = torch.empty_like(dcal)
    S.trans_vsrc(vsrc, (encobs - dcal).contiguous())
    g64 = torch.zeros(exi.shape, dtype=torch.float64, device="cuda")
    t64, _ = _timed(torch, lambda: m.calgradient_ess_f64(velinit, encsrc.double(), vsrc.double(), g64))
    errs = {}
    b = s.nb + 6   # the unmasked interior: [b, nxpad-b) x [6, nzpad-b)

    def inner(a):
        return a[b:a.shape[0] - b, 6:a.shape[1] - b]

    def rel(a):
        return float(((inner(a).double() - inner(g64)).norm() / inner(g64).norm()).item())

    inner_errs, grad_s = {}, {}
    for name, fmt in (("f32", S.STRIP_F32), ("f16", S.STRIP_F16), ("bf16", S.STRIP_BF16)):
        m.set_strip_format(fmt)
        g = torch.zeros(exi.shape, device="cuda")
        m.calgradient_ess(encsrc, vsrc, g)
        errs[name] = float(((g.double() - g64).norm() / g64.norm()).item())
        inner_errs["strips_" + name] = rel(g)
        if name == "f32":
            grad_s["strips_f32"], _ = _timed(torch, lambda: m.calgradient_ess(encsrc, vsrc, g.zero_()))
    m.set_strip_format(S.STRIP_F32)
    for name, fmt in (("f32", S.STRIP_F32), ("f16", S.STRIP_F16), ("bf16", S.STRIP_BF16)):
        m.set_reconstruction(S.RECON_SNAPSHOTS, 64, fmt)
        g = torch.zeros(exi.shape, device="cuda")
        m.calgradient_ess(encsrc, vsrc, g)
        inner_errs["snapshots_" + name] = rel(g)
        if name == "f32":
            grad_s["snapshots_f32"], _ = _timed(torch, lambda: m.calgradient_ess(encsrc, vsrc, g.zero_()))
    m.set_reconstruction(S.RECON_STRIPS)
    dobs_h = dobs.cpu().numpy()
    del dobs, encobs
    f = S.EssFwiFramework(m, exi, s.vmin, s.vmax, s.nita, s.maxdv, wlt_h, dobs_h)
    t_first, _ = _timed(torch, lambda: f.epoch(0))
    ts = []
    for it in range(1, iters + 1):
        t, _ = _timed(torch, lambda: f.epoch(it))
        ts.append(t)
    per = sum(ts) / len(ts)
    return {"workload": "encoded-source FWI: 96 shots of 301x921 (993x343 padded) as one supershot, nt 4000, "
                        "dt 1 ms, 15 Hz, codes re-drawn each iteration",
            "iterations_timed": len(ts), "s_per_iteration": per, "fifty_iterations_s": 50 * per,
            "gpu_first_epoch_s": t_first, "trials_last": f.lastTrials(),
            "gradient_rel_l2_vs_f64": errs, "f64_gradient_s": t64,
            "interior_gradient_rel_l2_vs_f64": inner_errs, "supershot_gradient_s": grad_s,
            "strips": "FP32 during the timed iterations; FP16/BF16 scaled strips in the error figures",
            "snapshots": "checkpoint snapshots of both fields every 64 steps (FP32 or scaled FP16/BF16), each "
                         "segment re-run forward in the backward sweep; errors on the unmasked interior"}


def record_enkf(torch, arith, tuning, cpu, members=64):
    """Ensemble Kalman FWI analysis: 201 x 461 (243 x 533 padded), 20 m,
    nt 3000, dt 2 ms, 16 shots encoded into one supershot per member
    (EnkfAnalyze::calGainMatrix's HA loop, enkfanalyze.cpp:207-236) for 64
    members = initial model + Gaussian random fields (200 m, 100 m/s);
    observed data with Gaussian noise at 1 % of each trace's RMS.  Timed:
    the batched member forward (HA), the FP64 gain (cross products,
    factorisation, products) and the member update."""
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    from swfwi_b200.enfwi import vel_recover, vel_trans
    s = sv.config("enkf")
    vt = sv.layered_model(s.nx, s.nz, seed=2024)
    vi = sv.smooth(vt, 15.0).astype(np.float32)
    m = S.Damp4t10d.from_survey(s, arith=arith)
    m.set_tuning(**tuning)
    ext, exi = m.expandDomain(vt), m.expandDomain(vi)
    wlt_h = S.ricker_wavelet(s.nt, s.fm, s.dt)
    wlt = torch.from_numpy(wlt_h).cuda()
    vel = torch.from_numpy(ext).cuda()
    m.bindVelocity(vel)
    dobs = torch.zeros((s.ns, s.nt, s.ng), device="cuda")
    m.forward_batch(wlt, dobs, np.arange(s.ns, dtype=np.int32))
    g = torch.Generator(device="cuda").manual_seed(7)
    rms = dobs.pow(2).mean(dim=1, keepdim=True).sqrt()
    dobs += 0.01 * rms * torch.randn(dobs.shape, device="cuda", generator=g)
    v0 = vel_recover(exi, s.dx, s.dt)
    nxpad, nzpad = exi.shape
    vels = np.stack([vel_trans(v0 + sv.gaussian_random_field(nxpad, nzpad, s.dx, 200.0, 100.0, seed=100 + i),
                               s.dx, s.dt) for i in range(members)])
    vels = torch.from_numpy(vels).cuda()
    ea = S.EnkfAnalyze(m, wlt, dobs, sigfac=0.5)
    codes = torch.from_numpy(S.random_codes(2, s.ns)).cuda()
    encsrc = torch.empty((s.nt, s.ns), device="cuda")
    S.encode_source(encsrc, wlt, codes)
    encobs = torch.empty((s.nt, s.ng), device="cuda")
    S.encode_obs(encobs, dobs, codes)
    d = encobs.t().contiguous().reshape(-1)
    hona = torch.empty((members, s.ng * s.nt), device="cuda")
    m.ess_forward_members(encsrc, vels, hona)            # warm-up
    t_ha, _ = _timed(torch, lambda: m.ess_forward_members(encsrc, vels, hona))
    t_gain, (t4, sigma, clip) = _timed(torch, lambda: S.enkf_gain_matrix(hona, d, None, 0.5, 0.0, 1))
    t_upd, _ = _timed(torch, lambda: S.enkf_update(vels.reshape(members, -1), t4, s.dx, s.dt))
    rows = s.ng * s.nt
    pts = (nxpad - 12) * (nzpad - 12) * s.nt * members
    rec = {"workload": f"EnKF analysis: {members} members x one 16-shot supershot of 201x461 (243x533 padded), "
                       "nt 3000, dt 2 ms; FP32 member modelling, FP64 analysis",
           "members": members, "ha_s": t_ha, "ha_gpts": pts / t_ha / 1e9,
           "gain_s": t_gain, "update_s": t_upd, "clip": int(clip),
           "cross_products_gflop": 6.0 * members * members * rows / 1e9,
           "gain_fp64_gflops": 6.0 * members * members * rows / t_gain / 1e9}
    if cpu:
        import oracle
        if oracle.available():
            R = oracle.RefLib()
            ntc = 600
            ss = s.scaled(nt=ntc)
            M = R.model(ss)
            M.bind_velocity(exi)
            enc = np.ascontiguousarray(np.outer(S.ricker_wavelet(ntc, s.fm, s.dt),
                                                S.random_codes(2, s.ns)).astype(np.float32))
            tf, _ = _cpu_timed(lambda: M.ess_forward(enc))
            cpu_ha = tf * (s.nt / ntc) * members
            rec["cpu"] = {"ha_s": cpu_ha, "kind": "reference", "cores": _cores(),
                          "basis": f"extrapolated: {members} members x the reference's EssForwardModeling of "
                                   f"one member timed at nt {ntc} ({tf:.2f} s) x {s.nt}/{ntc}; the "
                                   "reference's analysis needs MPI and LAPACK and is not timed"}
            rec["ha_speedup_vs_cpu"] = cpu_ha / t_ha
    return rec


def record_lsrtm(torch, cpu=True):
    """The LSRTM operator (src/unused/prtm2d.cpp) on the plain-FWI survey
    (151 x 461, 25 m, dt 2 ms, nt 2000, 20 shots, 461 receivers, 30-cell
    sponge) with a layered model: Born modelling and migration (the
    reference's, and the exact transpose of Born) in FAST arithmetic, all
    shots in one batch.  Work unit: grid-point updates of the padded fields
    (Born: source and scattered field, 2 per point per step; migration: the
    source field forward, then its reconstruction and the receiver field, 3
    per point per step).  Parity: the dot-product test of Born and its exact
    transpose on this survey."""
    import swfwi_b200 as S
    from swfwi_b200 import survey as sv
    s = sv.config("fwi")
    vt = sv.layered_model(s.nx, s.nz, seed=2024)
    vel = torch.from_numpy(np.ascontiguousarray(vt)).cuda()
    kw = dict(dz=s.dx, dx=s.dx, dt=s.dt, amp=1.0, fm=s.fm, nb=s.nb, nt=s.nt, ng=s.ng, sxbeg=s.sxbeg, szbeg=1,
              jsx=s.jsx, jsz=0, gxbeg=0, gzbeg=1, jgx=1, jgz=0)
    op = S.Prtm2d(vel, ns=s.ns, arith=S.ARITH_FAST, **kw)
    g = torch.Generator(device="cuda").manual_seed(3)
    mod = torch.randn((s.nx, s.nz), device="cuda", generator=g)
    dat = torch.randn((s.ns, s.ng, s.nt), device="cuda", generator=g)
    born = torch.empty_like(dat)
    img = torch.empty_like(mod)
    op.lop(False, False, mod, born)                        # warm-up
    t_born, _ = _timed(torch, lambda: op.lop(False, False, mod, born))
    t_mig, _ = _timed(torch, lambda: op.lop(True, False, img, dat))
    op.set_adjoint(S.PRTM_ADJ_EXACT)
    t_adj, _ = _timed(torch, lambda: op.lop(True, False, img, dat))
    a = float(torch.dot(born.double().ravel(), dat.double().ravel()))
    b = float(torch.dot(mod.double().ravel(), img.double().ravel()))
    op.close()
    pts = (s.nx + 2 * s.nb) * (s.nz + 2 * s.nb) * s.nt * s.ns
    rec = {"workload": f"LSRTM operator, {s.ns} shots of {s.nx}x{s.nz} ({s.nx + 2 * s.nb}x{s.nz + 2 * s.nb} "
                       f"padded), nt {s.nt}, {s.ng} receivers; FAST arithmetic, one batch",
           "born_s": t_born, "born_gpts": 2 * pts / t_born / 1e9,
           "migration_s": t_mig, "migration_gpts": 3 * pts / t_mig / 1e9,
           "exact_adjoint_s": t_adj, "exact_adjoint_gpts": 3 * pts / t_adj / 1e9,
           "unit": "Gpts/s of padded-field point updates (Born 2, migration 3 per point per step)",
           # FP32 over 2000 steps, the source field rebuilt backwards from
           # its ring: exact in exact arithmetic, 1e-4 in float
           "dot_product": {"lm_d": a, "m_ltd": b, "rel": abs(a - b) / abs(a), "tolerance": 1e-4,
                           "ok": abs(a - b) <= 1e-4 * abs(a)}}
    if cpu:
        import oracle
        if os.path.exists(os.path.join(oracle.REF_DIR, "libprtm_ref.so")):
            r = oracle.PrtmRef(vt, ns=1, **kw)
            m1 = mod.cpu().numpy()
            d1 = np.zeros((1, s.ng, s.nt), np.float32)
            tc, _ = _cpu_timed(lambda: r.lop(0, 0, m1, d1))
            r.close()
            rec["cpu"] = {"born_s": tc * s.ns, "kind": "reference", "cores": _cores(),
                          "basis": f"the reference's prtm2d_lop Born branch (compiled in place, OpenMP) for one "
                                   f"shot ({tc:.2f} s) x {s.ns} shots"}
            rec["born_speedup_vs_cpu"] = tc * s.ns / t_born
    return rec


def _cores():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def network_flops(layers, N, H, W):
    """Multiply-add FLOPs of one forward of the preconditioner network and of
    one training step (forward, weight gradient, data gradient of every conv
    but the first) on N images of H x W; layers: the library's layer table
    [(cin, cout, w_off, b_off)] (14 convs, then the 1x1 output)."""
    P0 = N * H * W
    level = [0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0]
    fwd = sum(2.0 * (P0 // 4 ** level[l]) * 9 * ci * co for l, (ci, co, _, _) in enumerate(layers[:-1]))
    fwd += 2.0 * P0 * layers[-1][0]
    first = 2.0 * P0 * 9 * layers[0][0] * layers[0][1]
    return fwd, 3 * fwd - first


def run_learned_mode(args):
    print(json.dumps(learned_record(args, verbose=True)))
    return 0


def learned_record(args, verbose=False):
    """FWI wall-clock to equal model error, learned vs plain: train the
    preconditioner on plain FWI runs over seeded models, then on each
    held-out model run plain FWI for its epoch budget and learned FWI until
    it reaches the lowest model error plain reached.  value: the geometric
    mean over the held-out models of plain seconds / learned seconds, with
    every model's own figure beside it.  Also times the network's kernels."""
    import math
    import torch
    from swfwi_b200 import precond as P
    s = P.demo_survey(nz=args.learned_nz, nx=args.learned_nx, nt=args.learned_nt,
                      ns=args.learned_shots).scaled(maxdv=100.0)
    net, st = P.train_from_plain(s, range(100, 100 + args.learned_models), args.learned_iters,
                                 args.learned_epochs, batch=16, horizon=args.learned_horizon)
    if verbose:
        print(json.dumps({"training": st}), file=sys.stderr, flush=True)
    tests = []
    for seed in args.learned_test_seeds:
        r = P.compare(s, net, seed, args.learned_iters, min_decrease=args.learned_min_decrease)
        reached = r["learned_s"] is not None
        # a learned run that never reaches the target counts with its whole
        # run time: an upper bound on its speed-up
        learned_s = r["learned_s"] if reached else r["learned_history"][-1][0]
        sp = r["plain_s"] / learned_s
        tests.append({"seed": seed, "speedup": sp, "reached": reached, "plain_s": r["plain_s"],
                      "learned_s": learned_s,
                      "target_model_error": r["target_error"], "initial_model_error": r["initial_error"],
                      "learned_steps": {"tried": r["learned_stats"][1], "accepted": r["learned_stats"][2]},
                      "plain_history": [[round(a, 3), b] for a, b, _, _ in r["plain_history"]],
                      "learned_history": [[round(a, 3), b, bool(d)] for a, b, _, d in r["learned_history"]]})
        if verbose:
            print(json.dumps({k: v for k, v in tests[-1].items() if "history" not in k}), file=sys.stderr,
                  flush=True)
    sps = [t["speedup"] for t in tests]
    value = math.exp(sum(math.log(x) for x in sps) / len(sps))
    H, W = P.image_shape(P.Damp4t10d.from_survey(s))
    network = time_network(net, 16, H, W)
    line = {
        "metric": "FWI wall-clock to equal model L2, learned vs plain",
        "value": value, "unit": "x (plain seconds / learned seconds, geometric mean over held-out models; "
                                "a learned run that never reaches the target counts with its whole time)",
        "higher_is_better": True, "n_gpus": 1, "dtype": "f32 wavefields, bf16 network (f32 accumulate)",
        "data": "synthetic",
        "model_error": "relative L2 of the interior velocity (m/s) against the true model; target: the "
                       "lowest error the plain run reaches in its epoch budget",
        "config": {"workload": f"learned-preconditioned FWI, {s.nx}x{s.nz} grid (dx {s.dx} m), nt={s.nt}, "
                               f"{s.ns} shots, {s.fm} Hz Ricker; seeded gradient+anomaly models",
                   "train_models": args.learned_models, "plain_iters": args.learned_iters,
                   "train_epochs": args.learned_epochs, "maxdv": s.maxdv,
                   "learned_min_decrease": args.learned_min_decrease,
                   "target_horizon": args.learned_horizon,
                   "test_seeds": list(args.learned_test_seeds)},
        "training": st, "tests": tests, "network": network,
    }
    return line


def time_network(net, N, H, W, reps=10):
    """The preconditioner's kernels on a batch of N images of H x W: forward
    and training step (forward, backward, Adam) timed with CUDA events on the
    launching stream, with the tensor-core throughput of the training step."""
    import torch
    x = torch.randn((N, H, W, 3), device="cuda")
    t = torch.randn((N, H, W), device="cuda")
    for _ in range(3):
        net.forward(x)
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        net.forward(x)
    e1.record(st)
    e1.synchronize()
    fwd_ms = e0.elapsed_time(e1) / reps
    saved = net.params()
    for _ in range(3):   # first use: kernel loading, attributes, scratch
        net.train_step(x, t, 1e-9)
    e0.record(st)
    for _ in range(reps):
        net.train_step(x, t, 1e-9)
    e1.record(st)
    e1.synchronize()
    train_ms = e0.elapsed_time(e1) / reps
    net.set_params(saved)
    fwd_flop, train_flop = network_flops(net.layers(), N, H, W)
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, peak_basis = float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        peak, peak_basis = 1590.0, "fallback"
    return {"image": [H, W], "batch": N, "forward_ms": fwd_ms, "train_step_ms": train_ms,
            "forward_gflop": fwd_flop / 1e9, "train_gflop": train_flop / 1e9,
            "forward_tflops": fwd_flop / fwd_ms / 1e9, "train_tflops": train_flop / train_ms / 1e9,
            "bf16_peak_tflops": peak, "peak_basis": peak_basis,
            "train_frac": train_flop / train_ms / 1e9 / peak}


def run_network_mode(args):
    """The preconditioner's kernels alone (a seeded network, random images of
    the learned workload's interior): the small case for ncu."""
    import torch
    from swfwi_b200 import precond as P
    s = P.demo_survey(nz=args.learned_nz, nx=args.learned_nx, nt=args.learned_nt, ns=args.learned_shots)
    H, W = P.image_shape(P.Damp4t10d.from_survey(s))
    torch.manual_seed(0)
    net = P.Preconditioner()
    print(json.dumps({"mode": "network", **time_network(net, 16, H, W)}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--arith", default="fast", choices=["ref", "fast"],
                    help="fast: FP32 with FMA (seismograms within 1e-5, gradients within 1e-4 of the "
                         "reference); ref: the reference's rounding, bit-identical")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the records of the other workloads (plain FWI iteration, encoded-source "
                         "FWI, EnKF analysis, LSRTM operator, learned vs plain FWI)")
    ap.add_argument("--ess-iters", type=int, default=3, help="timed encoded-source FWI iterations")
    ap.add_argument("--no-learned", action="store_true",
                    help="leave the learned-vs-plain record (about four minutes) out of the configs")
    ap.add_argument("--mode", default="bench", choices=["bench", "kernel", "tune", "learned", "network"],
                    help="kernel: short 96-shot batched forward (the small case for ncu); "
                         "tune: print the autotuner's table; learned: FWI wall-clock to equal model "
                         "error, learned preconditioner vs plain")
    ap.add_argument("--learned-models", type=int, default=16, help="training models of --mode learned")
    ap.add_argument("--learned-iters", type=int, default=30, help="plain epochs per training/test run")
    ap.add_argument("--learned-epochs", type=int, default=100, help="training epochs of the network")
    ap.add_argument("--learned-nx", type=int, default=480)
    ap.add_argument("--learned-nz", type=int, default=160)
    ap.add_argument("--learned-nt", type=int, default=2000)
    ap.add_argument("--learned-shots", type=int, default=24)
    ap.add_argument("--learned-test-seeds", type=int, nargs="+", default=[200, 201, 202])
    ap.add_argument("--learned-horizon", type=int, default=None,
                    help="training target: the velocity this many plain epochs ahead (default: the run's end)")
    ap.add_argument("--learned-min-decrease", type=float, default=0.02,
                    help="a learned step is kept only if it lowers the objective by this fraction")
    ap.add_argument("--nt", type=int, default=24, help="steps of the kernel/tune modes")
    ap.add_argument("--tuning", default="", help="stencil launch shape as JSON (skips the autotuner)")
    ap.add_argument("--fuse", default="off", choices=["on", "off"],
                    help="fused backward time loop (source subtraction, imaging and residual injection "
                         "inside the step kernels)")
    ap.add_argument("--strips", default="f32", choices=["f32", "f16", "bf16"],
                    help="storage of the boundary strips the gradient saves")
    ap.add_argument("--workload-nt", type=int, default=0,
                    help="cut the time axis to this many steps (a short run for the ncu launch list; "
                         "not the benchmark workload)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "learned":
        return run_learned_mode(args)
    if args.mode == "network":
        return run_network_mode(args)
    if args.mode != "bench":
        return run_kernel_mode(args)

    import torch
    import swfwi_b200 as S
    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    arith = S.ARITH_REF if args.arith == "ref" else S.ARITH_FAST
    s, m, exi, exi_h, wlt, wlt_h, dobs, ids = setup_workload(torch, arith, args.workload_nt)
    nxpad, nzpad, ns, ngmax, nt = m.dims()
    from swfwi_b200 import autotune
    tuning = dict(autotune.DEFAULT)
    if args.tuning:
        tuning = json.loads(args.tuning)
    elif not args.no_tune:
        tuning, _ = autotune.tune(s, exi_h, arith)
    m.set_tuning(**tuning)
    m.set_fusion(args.fuse == "on")
    m.set_strip_format({"f32": S.STRIP_F32, "f16": S.STRIP_F16, "bf16": S.STRIP_BF16}[args.strips])
    grad = torch.zeros((nxpad, nzpad), dtype=torch.float32, device="cuda")

    # the time loops replay as CUDA graphs (mode 2: captured in the first
    # warm-up step); the stencil timing is part of the captured graphs, so
    # it is on from the start
    m.set_graphs(2)
    S.stats_enable_step_timing(TIMING_PERIOD)
    for _ in range(max(args.warmup, 0)):
        m.gradient_batch(wlt, dobs, ids, grad)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()

    S.stats_reset()
    # every launch's work counted, every TIMING_PERIOD-th stencil launch timed
    # with CUDA events (event nodes in the replayed graphs)
    clk = ClockSampler(local)
    clk.start()
    stream = torch.cuda.current_stream()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()       # ncu --profile-from-start off sees the timed steps only
    ev0.record(stream)
    objs = None
    for _ in range(args.steps):
        objs = m.gradient_batch(wlt, dobs, ids, grad)
    ev1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    barrier()
    clocks = clk.stop()
    ms = ev0.elapsed_time(ev1)
    st = S.stats_read()
    S.stats_enable_step_timing(False)
    ms_max = max_over_ranks(ms, dist)
    updates_rank = st["step_point_updates"]
    value = replica_value(updates_rank, world, ms_max * 1e-3)

    # dominant kernel: the stencil step, timed per launch with CUDA events
    peak, peak_kind = measured_peaks()
    timed = max(st["step_timed_launches"], 1)
    avg_launch_s = st["step_ms"] * 1e-3 / timed
    bytes_per_launch = st["step_bytes"] / max(st["step_launches"], 1)
    step_gbs = bytes_per_launch / avg_launch_s / 1e9 if st["step_ms"] > 0 else 0.0
    per_launch_pts = st["step_point_updates"] / max(st["step_launches"], 1)
    tpp = traffic_per_point(tuning.get("kernel", 1))
    roofline = {"bound": "hbm", "achieved": step_gbs, "peak": peak, "unit": "GB/s",
                "frac": step_gbs / peak, "peak_basis": peak_kind,
                "traffic": (tpp * per_launch_pts) if tpp else None,
                "kernel": {1: "fd_step_ws", 5: "fd_step_rq", 6: "fd_step_rq2"}.get(tuning.get("kernel", 6)),
                "launches": st["step_launches"], "timed_launches": st["step_timed_launches"],
                "timing": f"CUDA events around every {TIMING_PERIOD}th stencil launch of the timed region (event "
                          "nodes inside the replayed time-loop graphs)",
                "avg_launch_us": avg_launch_s * 1e6,
                "bytes_per_launch": bytes_per_launch,
                "stencil_share_of_step": avg_launch_s * st["step_launches"] / (ms * 1e-3) if ms > 0 else None}

    # end to end through the C ABI from pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        dobs_h = torch.empty(dobs.shape, dtype=torch.float32, pin_memory=True)
        dobs_h.copy_(dobs.cpu())
        exi_p = torch.from_numpy(exi_h).pin_memory()
        wlt_p = torch.from_numpy(wlt_h).pin_memory()
        grad_p = torch.empty((nxpad, nzpad), dtype=torch.float32, pin_memory=True)
        # counts the point-updates, times one launch; set before the warm-up
        # call, which captures the loops' graphs with this setting
        S.stats_enable_step_timing(1 << 30)
        m.gradient_host(exi_p.numpy(), wlt_p.numpy(), dobs_h.numpy(), ids, grad_p.numpy())
        S.stats_reset()
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            m.gradient_host(exi_p.numpy(), wlt_p.numpy(), dobs_h.numpy(), ids, grad_p.numpy())
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        st2 = S.stats_read()
        S.stats_enable_step_timing(False)
        dt = max_over_ranks(dt, dist)
        h2d = exi_p.numel() * 4 + wlt_p.numel() * 4 + dobs_h.numel() * 4
        e2e = {"value": replica_value(st2["step_point_updates"], world, dt), "unit": "Gpts/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(grad_p.numel() * 4 + 8 * ns),
               "ms_per_step": dt / args.e2e_steps * 1e3}
        m.bindVelocity(exi)

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            info = cpu_reference_sample()
            if info:
                cpu = {"value": info["updates"] / info["seconds"] / 1e9, "unit": "Gpts/s",
                       "cores": info["cores"], "kind": "reference", "sample": info["sample"],
                       "seconds": info["seconds"]}
                parity = parity_of_sample(torch, arith, tuning, info)
                ab = cpu_reference_sample(nt_sample=CPU_SAMPLE_NT_ASBUILT, asbuilt=True)
                cpu["as_built"] = {"value": ab["updates"] / ab["seconds"] / 1e9, "unit": "Gpts/s",
                                   "cores": ab["cores"], "sample": ab["sample"], "seconds": ab["seconds"]}
        except Exception as e:   # the baseline is reported, never required
            cpu = {"value": None, "unit": "Gpts/s", "cores": 0, "kind": "reference",
                   "sample": f"failed: {e}"}

    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        configs = {}
        # the records run other grids and batch sizes: the tuned kernel with
        # the automatic task length, which sizes the tasks for each grid (a
        # row count tuned on this grid leaves small grids with few tasks)
        rec_tuning = dict(tuning, rows_per_cta=0)
        for key, fn in (("fwi_iteration_151x461", lambda: record_fwi_iteration(torch, arith, rec_tuning,
                                                                                not args.no_cpu_baseline)),
                        ("encoded_fwi_301x921", lambda: record_encoded(torch, arith, rec_tuning, args.ess_iters)),
                        ("enkf_201x461", lambda: record_enkf(torch, arith, rec_tuning, not args.no_cpu_baseline)),
                        ("lsrtm_151x461", lambda: record_lsrtm(torch, not args.no_cpu_baseline)),
                        ("learned_fwi", lambda: None if args.no_learned else learned_record(args))):
            try:
                configs[key] = fn()
            except Exception as e:   # reported, never required
                configs[key] = {"failed": f"{type(e).__name__}: {e}"}
            torch.cuda.synchronize()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Gpts/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "batched FWI gradient, 96 shots, 301x921 grid (993x337 padded), "
                                       f"nt={nt}, uneven spreads 200-921"
                                       + (" (REDUCED time axis: not the benchmark)" if args.workload_nt else ""),
                           "shots": int(ns), "nt": int(nt), "grid": [int(nxpad), int(nzpad)],
                           "arith": args.arith, "strips": args.strips, "fused": args.fuse == "on", "tuning": tuning,
                           "point_updates_per_step": updates_rank / args.steps,
                           "l2": "inputs larger than L2 (strips 14 GB, fields 0.5 GB): no flush",
                           "parallelism": f"replicas{world}",
                           "objective_last_step": float(np.sum(objs)) if objs is not None else None},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "parity": parity,
                "gpu_launches": int(st["kernel_launches"]), "clocks": clocks, "configs": configs}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
