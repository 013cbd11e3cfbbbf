#!/usr/bin/env python
"""Benchmark of the operator-method pricing path on B200.

Workload (one step = one full lattice solve): the stochastic-volatility lattice with
48 vol states x 128 log-spot states (d = 6144), dt0 = 2^-16, 14 squarings to P(0.25),
chaining to 16 quarterly maturities, backward induction of 128 call payoffs with FP64
discounting -> 2048 quotes.  The generator is rebuilt on the device every step.

Metric: priced quotes per second, split-BF16 tensor-core path (default) at <= 1e-5
absolute error versus an FP64 solve of the same lattice; the plain FP32 path and the
error of both are reported in the same line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--mode bf16x3|fp32]

Under torchrun every rank solves its own replica (the lattice does not shard; "replicas
only"), timing is the max over ranks, value is the job total.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SV = dict(nx=128, nv=48, x_lo=0.05, x_hi=5.0, v_lo=0.05, v_hi=1.0, rate=0.03, kappa=2.0, theta=0.04, xi=0.6, rho=-0.7)
PERIOD, NMAT, NK, DT0 = 0.25, 16, 128, 2.0 ** -16
NITER_SV = 14  # squarings to P(PERIOD) at dt0 (the plan rule; checked against the plan at run time)
SV_METRIC = "priced quotes/sec at <=1e-5 abs err vs FP64 (split-BF16 tensor-core lattice vs plain FP32)"


def sv_config(mode: str, world: int) -> dict:
    """The headline workload's config, shared by both arms of the bench."""
    return {"workload": "SV lattice 48 vol x 128 spot = 6144 states, dt0=2^-16, 14 squarings + 15 chains, "
                        "128 strikes x 16 quarterly maturities (2048 quotes/solve)",
            "d": SV["nx"] * SV["nv"], "niter": NITER_SV, "nmat": NMAT, "nK": NK, "mode": mode,
            "parallelism": f"replicas x{world}", "l2": "operands 151-302 MB per matrix > 126 MB L2"}
STRIKES = [0.5 + j / 127.0 for j in range(NK)]


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], d["bf16_tflops"], d.get("bf16_tflops_sustained", d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.index, self.proc, self.f = index, None, None

    def __enter__(self):
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def fp64_reference_quotes(lat, plan, torch):
    """Plain FP64 restatement of the solve with torch on the device (accuracy check only,
    outside the timed region): dense L from the ELL generator, (I + dt L)^(2^niter) with
    row renormalisation, chaining, payoff induction, discounting."""
    d = lat.d
    dev = lat.device
    cols = lat.cols.view(d, -1).long()
    vals = lat.vals.view(d, -1)
    L = torch.zeros(d, d, dtype=torch.float64, device=dev)
    mask = cols >= 0
    rows = torch.arange(d, device=dev).unsqueeze(1).expand_as(cols)
    L.index_put_((rows[mask], cols[mask]), vals[mask], accumulate=True)
    P = torch.eye(d, dtype=torch.float64, device=dev) + plan.dt * L
    del L
    for _ in range(plan.niter):
        P = P @ P
        P /= P.sum(dim=1, keepdim=True)
    K = torch.tensor(STRIKES, dtype=torch.float64, device=dev)
    G = torch.clamp(lat.x.unsqueeze(1) - K.unsqueeze(0), min=0.0)
    out = []
    Pm = P
    for m in range(1, NMAT + 1):
        if m > 1:
            Pm = Pm @ P
            Pm /= Pm.sum(dim=1, keepdim=True)
        out.append(math.exp(-lat.rate * PERIOD * m) * (Pm[lat.y0] @ G))
    return torch.stack(out)


def fp32_cublas_solve(lat, plan, strikes, torch, out, nmat=NMAT, period=PERIOD):
    """The plain-FP32 comparison arm on cuBLAS (TF32 off): U0 = I + dt L in FP32 from the
    ELL generator, niter squarings and the chain products as cuBLAS SGEMMs, each followed by
    the FP64 row renormalisation that the 1e-5 bar needs (FP64 row sums, FP32 scaling),
    pricing P(T_m) G in FP32 and the FP64 discount.  Writes quotes [nmat, nK] into out."""
    d = lat.d
    dev = lat.device
    cols = lat.cols.view(d, -1).long()
    vals = lat.vals.view(d, -1)
    mask = cols >= 0
    rows = torch.arange(d, device=dev).unsqueeze(1).expand_as(cols)
    P = torch.zeros(d, d, dtype=torch.float32, device=dev)
    P.index_put_((rows[mask], cols[mask]), (plan.dt * vals[mask]).float(), accumulate=True)
    P.diagonal().add_(1.0)
    T = torch.empty_like(P)

    def renorm(X):
        s = X.sum(dim=1, dtype=torch.float64)
        X.mul_((1.0 / s).float().unsqueeze(1))

    for _ in range(plan.niter):
        torch.mm(P, P, out=T)
        P, T = T, P
        renorm(P)
    G = torch.clamp(lat.x.unsqueeze(1) - strikes.unsqueeze(0), min=0.0).float()
    Pm = P.clone()
    for m in range(1, nmat + 1):
        if m > 1:
            torch.mm(Pm, P, out=T)
            Pm, T = T, Pm
            renorm(Pm)
        out[m - 1] = math.exp(-lat.rate * period * m) * (Pm[lat.y0] @ G).double()
    return out


def run_b200(args, rank, world, local_rank):
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import MODES, Lattice, bind_stream

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev)
    bind_stream(dev)
    mode = MODES[args.mode]
    sv = dict(SV)
    sv["rho"] = SV["rho"] + 0.001 * rank  # independent replica per rank
    lat = Lattice.stoch_vol(**sv, device=dev)
    plan = lat.plan(PERIOD, DT0)
    if plan.niter != NITER_SV:
        raise SystemExit(f"plan gives {plan.niter} squarings, the workload states {NITER_SV}")
    strikes = torch.tensor(STRIKES, dtype=torch.float64, device=dev)
    ws = lat.workspace(NK, mode)
    quotes = torch.empty(NMAT, NK, dtype=torch.float64, device=dev)
    desc = lat.desc(plan, PERIOD, NMAT, strikes)
    d = lat.d

    def build_generator():
        _lib.call("opb_sv_generator_ell", sv["nx"], sv["nv"], sv["x_lo"], sv["x_hi"], sv["v_lo"], sv["v_hi"],
                  sv["rate"], sv["kappa"], sv["theta"], sv["xi"], sv["rho"], lat.cols.data_ptr(),
                  lat.vals.data_ptr(), lat.x.data_ptr())

    def step():
        build_generator()
        _lib.call("opb_lattice_solve", C.byref(desc), mode, ws.data_ptr(), ws.numel(), quotes.data_ptr(), None)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    assert lib.opb_tc_error() == 0

    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local_rank) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    clocks = clk.summary()

    # ---- end to end through the C ABI: pinned host strikes in, quotes out, every step
    h_strikes = torch.tensor(STRIKES, dtype=torch.float64).pin_memory()
    h_quotes = torch.empty(NMAT, NK, dtype=torch.float64).pin_memory()

    def e2e_step():
        strikes.copy_(h_strikes, non_blocking=True)
        step()
        h_quotes.copy_(quotes, non_blocking=True)

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / args.steps
    if dist:
        t = torch.tensor([ms_e2e], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())

    # ---- dominant kernel timed alone with CUDA events on the launching stream
    hbm, bf16_burst, bf16_sus, src = _peaks()
    kern = {}
    if mode in (MODES["bf16x3"], MODES["fp16x3"]):
        f16 = mode == MODES["fp16x3"]
        Ah = torch.empty(d, d, dtype=torch.float16 if f16 else torch.bfloat16, device=dev).normal_(0, 1e-3)
        Al = torch.empty_like(Ah).normal_(0, 1e-6)
        gemm_fn = "opb_gemm_f16x3_kn" if f16 else "opb_gemm_bf16x3_kn"
        X = torch.empty(d, d, dtype=torch.float32, device=dev).normal_()
        rs = torch.empty(lib.opb_gemm_bf16x3_nparts(d, d) * d, dtype=torch.float64, device=dev)
        args_g = (d, d, d, Ah.data_ptr(), Al.data_ptr(), d, Ah.data_ptr(), Al.data_ptr(), d, 1.0, X.data_ptr(), 2.0,
                  X.data_ptr(), d, rs.data_ptr())
        for _ in range(3):
            _lib.call(gemm_fn, *args_g)
        torch.cuda.synchronize()
        n_rep = 20
        e0.record(stream)
        for _ in range(n_rep):
            _lib.call(gemm_fn, *args_g)
        e1.record(stream)
        torch.cuda.synchronize()
        k_ms = e0.elapsed_time(e1) / n_rep
        mma_flops = 3 * 2.0 * d ** 3
        achieved = mma_flops / (k_ms * 1e-3) / 1e12
        # DRAM bytes (read + write) of one launch of this kernel at d = 6144 from an ncu
        # capture (dram__bytes_read.sum 940.9 MB + dram__bytes_write.sum 148.3 MB); the
        # algorithmic traffic is 4 BF16 operand reads + Cin read, C written = 16 d^2 + 8 d^2
        # bytes.
        traffic = 1089.2e6 if d == 6144 else None
        kern = {"bound": "tensor", "achieved": round(achieved, 1), "peak": bf16_burst, "unit": "TFLOP/s",
                "frac": round(achieved / bf16_burst, 4), "frac_of_sustained": round(achieved / bf16_sus, 4),
                "traffic": traffic, "traffic_unit": "DRAM bytes per launch",
                "algorithmic_bytes": 24.0 * d * d, "peak_source": f"{src} burst bf16",
                "kernel": "k_tc_gemm<256,3,pair,MN-major B> (E-form squaring on 2-CTA clusters, cta_group::2, "
                          f"{d}^3 x 3 {'FP16' if f16 else 'BF16'} products, B = E's own row-major parts)",
                "avg_launch_ms": round(k_ms, 4), "useful_tflops": round(achieved / 3, 1)}
        del Ah, Al, X, rs
    else:
        A = torch.empty(d, d, dtype=torch.float32, device=dev).uniform_()
        Cc = torch.empty_like(A)
        for _ in range(2):
            _lib.call("opb_sgemm_batched_rm", d, d, d, A.data_ptr(), 0, A.data_ptr(), 0, Cc.data_ptr(), 0, 1)
        torch.cuda.synchronize()
        n_rep = 5
        e0.record(stream)
        for _ in range(n_rep):
            _lib.call("opb_sgemm_batched_rm", d, d, d, A.data_ptr(), 0, A.data_ptr(), 0, Cc.data_ptr(), 0, 1)
        e1.record(stream)
        torch.cuda.synchronize()
        k_ms = e0.elapsed_time(e1) / n_rep
        achieved = 2.0 * d ** 3 / (k_ms * 1e-3) / 1e12
        kern = {"bound": "fp32-simt", "achieved": round(achieved, 2), "peak": 74.4, "unit": "TFLOP/s",
                "frac": round(achieved / 74.4, 4), "traffic": None,
                "peak_source": "nominal FP32 FMA (148 SM x 128 lanes x 2 x 1.965 GHz)",
                "kernel": "k_sgemm_rm (128x128 SIMT tile)", "avg_launch_ms": round(k_ms, 4)}
        del A, Cc

    # ---- accuracy of this step's quotes vs an FP64 solve of the same lattice
    step()
    torch.cuda.synchronize()
    q_ref = fp64_reference_quotes(lat, plan, torch)
    err = float((quotes - q_ref).abs().max().item())
    # the plain FP32 path on the same lattice (comparison arm), timed the same way
    extra = {}
    if args.compare and mode == MODES["bf16x3"]:
        m32 = MODES["fp32"]
        ws32 = lat.workspace(NK, m32)
        q32 = torch.empty_like(quotes)
        _lib.call("opb_lattice_solve", C.byref(desc), m32, ws32.data_ptr(), ws32.numel(), q32.data_ptr(), None)
        torch.cuda.synchronize()
        e0.record(stream)
        _lib.call("opb_lattice_solve", C.byref(desc), m32, ws32.data_ptr(), ws32.numel(), q32.data_ptr(), None)
        e1.record(stream)
        torch.cuda.synchronize()
        ms32 = e0.elapsed_time(e1)
        extra = {"fp32_quotes_per_s": round(NMAT * NK * world / (ms32 * 1e-3), 1), "fp32_ms_per_solve": round(ms32, 2),
                 "fp32_max_abs_err_vs_fp64": float((q32 - q_ref).abs().max().item()),
                 "speedup_vs_fp32": round(ms32 / ms, 2)}
        del ws32
        # context for the comparison arm: the library's SIMT FP32 product against cuBLAS
        # SGEMM (TF32 off) at the same size; the plain solve re-estimated with cuBLAS
        # products in place of the 29 SIMT ones
        A32 = torch.empty(d, d, dtype=torch.float32, device=dev).uniform_()
        C32 = torch.empty_like(A32)
        tf32 = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = False
        torch.mm(A32, A32, out=C32)
        t_cu = _time(lambda: torch.mm(A32, A32, out=C32), 5, stream, torch)
        torch.backends.cuda.matmul.allow_tf32 = tf32
        t_si = _time(lambda: _lib.call("opb_sgemm_batched_rm", d, d, d, A32.data_ptr(), 0, A32.data_ptr(), 0,
                                       C32.data_ptr(), 0, 1), 3, stream, torch)
        extra["fp32_gemm_context"] = {"simt_tflops": round(2.0 * d ** 3 / (t_si * 1e-3) / 1e12, 1),
                                      "cublas_sgemm_tflops": round(2.0 * d ** 3 / (t_cu * 1e-3) / 1e12, 1)}
        del A32, C32
        # the cuBLAS plain-FP32 solve, measured; "plain FP32" is the faster of the two arms
        qcu = torch.empty_like(quotes)
        torch.backends.cuda.matmul.allow_tf32 = False
        fp32_cublas_solve(lat, plan, strikes, torch, qcu)
        torch.cuda.synchronize()
        e0.record(stream)
        fp32_cublas_solve(lat, plan, strikes, torch, qcu)
        e1.record(stream)
        torch.cuda.synchronize()
        torch.backends.cuda.matmul.allow_tf32 = tf32
        ms_cu = e0.elapsed_time(e1)
        extra["fp32_cublas_quotes_per_s"] = round(NMAT * NK * world / (ms_cu * 1e-3), 1)
        extra["fp32_cublas_ms_per_solve"] = round(ms_cu, 2)
        extra["fp32_cublas_max_abs_err_vs_fp64"] = float((qcu - q_ref).abs().max().item())
        extra["speedup_vs_fp32_simt"] = extra["speedup_vs_fp32"]
        extra["speedup_vs_fp32_cublas"] = round(ms_cu / ms, 2)
        extra["speedup_vs_fp32"] = round(min(ms32, ms_cu) / ms, 2)
        extra["fp32_arm"] = "cublas" if ms_cu < ms32 else "simt"
        del qcu
        m16 = MODES["fp16x3"]
        ws16 = lat.workspace(NK, m16)
        q16 = torch.empty_like(quotes)
        _lib.call("opb_lattice_solve", C.byref(desc), m16, ws16.data_ptr(), ws16.numel(), q16.data_ptr(), None)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(3):
            _lib.call("opb_lattice_solve", C.byref(desc), m16, ws16.data_ptr(), ws16.numel(), q16.data_ptr(), None)
        e1.record(stream)
        torch.cuda.synchronize()
        ms16 = e0.elapsed_time(e1) / 3
        extra["fp16x3"] = {"quotes_per_s": round(NMAT * NK * world / (ms16 * 1e-3), 1),
                           "max_abs_err_vs_fp64": float((q16 - q_ref).abs().max().item())}
        del ws16

    quotes_per_step = NMAT * NK * world
    value = quotes_per_step / (ms * 1e-3)
    # gpu launches per step (library kernels): generator, E0 scatter, split, niter*(gemm+renorm),
    # add_identity, split, payoff, nmat*(price gemm + discount), (nmat-1)*(chain gemm + renorm)
    if mode == MODES["bf16x3"]:
        # ... + the generator's band (one block)
        launches = 1 + 1 + 1 + 1 + 2 * plan.niter + 1 + 1 + 1 + 2 * NMAT + 2 * (NMAT - 1)
    else:
        launches = 1 + 2 + (3 if mode == 1 else 1) * plan.niter + 1 + 2 * NMAT + (3 if mode == 1 else 1) * (NMAT - 1)
    out = {
        "metric": SV_METRIC,
        "value": round(value, 1), "unit": "quotes/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16x3->fp32 (fp64 renorm/discount)" if mode == 2 else "fp32", "data": "synthetic",
        "config": sv_config(args.mode, world),
        "max_abs_err_vs_fp64": err,
        "e2e": {"value": round(quotes_per_step / (ms_e2e * 1e-3), 1), "unit": "quotes/s",
                "h2d_bytes_per_step": NK * 8, "d2h_bytes_per_step": NMAT * NK * 8},
        "gpu_launches": launches * args.steps,
        "roofline": kern,
        "clocks": clocks,
    }
    out.update(extra)
    return out


SWEEP_METRIC = "priced quotes/sec, calibration sweep (512 LV lattices, one tensor-core launch per level)"


def sweep_summary(args):
    """Config 3 beside the headline: the 512 seeded local-vol lattices (seed 20260, n in
    256..2048 step 128, 32 strikes x 8 quarterly maturities = 131,072 quotes) solved by the
    batched split path in bf16x3 and fp16x3 (every squaring level of all lattices one
    persistent launch, the sweep replayed from a CUDA graph, autotuned tiles), each lattice's
    quotes against an FP64 solve of it (all 512), and the two plain-FP32 arms on the same
    lattices: cuBLAS SGEMM (TF32 off) with FP64 renormalisation, per lattice, and the
    library's SIMT FP32 solve per lattice.  The speed-up is against the faster FP32 arm."""
    import torch
    from oplib_b200.model import Batch, bind_stream, calibration_sweep
    dev = torch.device("cuda", 0)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    nlat, nmat, period, dt0 = 512, 8, 0.25, 2.0 ** -14
    strikes = [0.5 + j / 31.0 for j in range(32)]
    nq = nlat * nmat * len(strikes)
    t_all = time.perf_counter()
    lats, _ = calibration_sweep(nlat=nlat, device=dev)
    out, plans = {}, None
    for mode in ("bf16x3", "fp16x3"):
        b = Batch(lats, strikes, nmat, period, dt0, mode=mode, autotune=True)
        plans = b.plans
        q = torch.empty(nlat, nmat, len(strikes), dtype=torch.float64, device=dev)
        for _ in range(max(1, args.warmup)):
            b.execute(q)
        g = _graph(lambda: b.execute(q), dev, torch)
        g.replay()
        ms = _time(g.replay, max(3, args.steps), stream, torch)
        out[mode] = {"quotes_per_s": round(nq / (ms * 1e-3), 1), "ms_per_sweep": round(ms, 3),
                     "config_chosen": b.config, "launches_per_sweep": b.launches(), "q": q.clone()}
        del g, b, q
    K = torch.tensor(strikes, dtype=torch.float64, device=dev)
    ref = torch.stack([_fp64_lv_quotes(lat, pl, strikes, nmat, period, torch) for lat, pl in zip(lats, plans)])
    tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    qcu = torch.empty(nlat, nmat, len(strikes), dtype=torch.float64, device=dev)

    def cublas_sweep():
        for i, (lat, pl) in enumerate(zip(lats, plans)):
            fp32_cublas_solve(lat, pl, K, torch, qcu[i], nmat=nmat, period=period)

    cublas_sweep()
    ms_cu = _time(cublas_sweep, 1, stream, torch)
    torch.backends.cuda.matmul.allow_tf32 = tf32
    b32 = Batch(lats, strikes, nmat, period, dt0, mode="fp32", autotune=False)
    q32 = b32.execute()
    ms_si = _time(lambda: b32.execute(q32), 1, stream, torch)
    torch.cuda.synchronize()
    res = {"metric": SWEEP_METRIC, "unit": "quotes/s", "quotes_per_sweep": nq,
           "workload": f"{nlat} LV lattices (seed 20260), n in 256..2048 step 128, niter "
                       f"{min(p.niter for p in plans)}..{max(p.niter for p in plans)}, 32 strikes x {nmat} maturities; "
                       "CUDA-graph replay; error over every lattice against its FP64 solve"}
    for mode in ("bf16x3", "fp16x3"):
        o = out[mode]
        e = (o.pop("q") - ref).abs().amax(dim=(1, 2))
        o["max_abs_err_vs_fp64"] = float(e.max().item())
        o["lattices_above_1e-5"] = int((e > 1e-5).sum().item())
        res[mode] = o
    res["fp32_cublas"] = {"quotes_per_s": round(nq / (ms_cu * 1e-3), 1), "ms_per_sweep": round(ms_cu, 1),
                          "max_abs_err_vs_fp64": float((qcu - ref).abs().max().item())}
    res["fp32_simt"] = {"quotes_per_s": round(nq / (ms_si * 1e-3), 1), "ms_per_sweep": round(ms_si, 1),
                        "max_abs_err_vs_fp64": float((q32 - ref).abs().max().item())}
    fastest32 = min(ms_cu, ms_si)
    res["fp32_arm"] = "cublas" if ms_cu <= ms_si else "simt"
    for mode in ("bf16x3", "fp16x3"):
        res[mode]["speedup_vs_fp32"] = round(fastest32 / res[mode]["ms_per_sweep"], 2)
    res["wall_s"] = round(time.perf_counter() - t_all, 1)
    del b32, q32, qcu, ref
    torch.cuda.empty_cache()
    return res


def surrogate_summary(args):
    """Config 4 beside the headline: the ensemble surrogate trained in this run by the
    library's kernels on ~2^21 lattice quotes (2600 seeded local-vol lattices, n = 1024,
    solved by the batched split path), then 2^20 quotes inferred on the tensor cores with 4
    and with 2 members: quotes/s, the lattice's quotes/s for the same family, the fallback
    rate (ensemble spread > 5 bp), the accepted quotes' error against the lattice in bp, and
    the quotes/s with the fallback quotes' lattices re-solved by the batched sweep."""
    a = argparse.Namespace(**vars(args))
    a.epochs, a.members, a.train_lattices = 40, 4, 2600
    a.steps, a.warmup = max(3, args.steps), max(3, args.warmup)
    t0 = time.perf_counter()
    line = run_surrogate(a)
    keep = ["value", "ms_per_step", "lattice_quotes_per_s", "speedup_vs_lattice", "fallback_rate", "fallback_lattices",
            "test_quotes", "accepted_err_bp", "all_err_bp", "baseline_err_bp", "effective_quotes_per_s_with_fallback",
            "two_members", "train_seconds", "data_seconds"]
    res = {"metric": "surrogate quotes/s (ensemble of 4 MLPs on tensor cores), 2^20 quotes", "unit": "quotes/s",
           "config": line["config"]}
    res.update({k: line[k] for k in keep if k in line})
    res["quotes_per_s"] = res.pop("value")
    res["wall_s"] = round(time.perf_counter() - t0, 1)
    return res


def mc_summary(args):
    """Config 2 beside the headline: the Monte Carlo of the LV(512) lattice, 2^20 paths x 504
    daily steps, one MT19937 stream per path, barrier and Asian calls (one step = step-kernel
    build + cumulative rows + guide table as one CUDA graph, then the MC kernel)."""
    a = argparse.Namespace(**vars(args))
    a.steps, a.warmup, a.mc_steps, a.cpu = 5, 3, 504, False
    t0 = time.perf_counter()
    line = run_mc(a)
    keep = ["value", "unit", "ms_per_step", "mc_kernel_only", "with_state_output", "prices"]
    res = {"metric": line["metric"], "config": line["config"]["workload"]}
    res.update({k: line[k] for k in keep if k in line})
    res["path_steps_per_s"] = res.pop("value")
    res["wall_s"] = round(time.perf_counter() - t0, 1)
    return res


def _host_info():
    """Host threads and CPU model string (recorded with every CPU number)."""
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return os.cpu_count() or 1, model


class HostSolve:
    """The reference's host FP64 solve of the headline SV lattice (``oracle.HostSolveFP64``:
    U0 = I + dt L, 14 squarings and 15 chain products as torch-CPU/MKL DGEMMs, the payoff
    product with each P_m) on all host threads, one product ("stage") at a time; a solve is
    29 stages.  The generator (dense FP64, 302 MB) is built once, outside every timing,
    like the strikes.  Denormal operands are flushed to zero (torch.set_flush_denormal): the
    far corners of the middle squarings' operands underflow, and FP64 products with
    denormal operands run several times slower on x86; flushing them changes no price and
    makes this CPU baseline faster, not slower."""

    def __init__(self):
        import torch

        from oracle import oracle as O
        self.nth, self.model = _host_info()
        torch.set_num_threads(self.nth)
        self.ftz = bool(torch.set_flush_denormal(True))
        spec = O.SVSpec(nx=SV["nx"], nv=SV["nv"], x_lo=SV["x_lo"], x_hi=SV["x_hi"], v_lo=SV["v_lo"], v_hi=SV["v_hi"],
                        r=SV["rate"], kappa=SV["kappa"], theta=SV["theta"], xi=SV["xi"], rho=SV["rho"])
        L, x, _ = O.sv_generator(spec)
        niter, dt = O.plan_niter(L, PERIOD, DT0)
        self.hs = O.HostSolveFP64(torch.from_numpy(L), x, STRIKES, SV["rate"], PERIOD, NMAT, niter, dt)
        self.niter, self.stages, self.d = niter, self.hs.stages, L.shape[0]

    def solve(self, keep=()):
        """One whole solve; returns (seconds, values, {stage: its input state} for the stages in
        ``keep``)."""
        inputs, state = {}, {}
        t0 = time.perf_counter()
        for p in range(self.stages):
            if p in keep:
                inputs[p] = state
            state = self.hs.run(p, state)
        t = time.perf_counter() - t0
        return t, self.hs.values(state), inputs

    def positions(self, k: int):
        """k stage positions spread evenly over a solve (all of them, cyclically, if k > 29), so
        that a sample of k stages weighs the solve's cheap and dear products as the solve does."""
        return [int((i + 0.5) * self.stages / k) % self.stages if k < self.stages else i % self.stages
                for i in range(k)]

    def run_stage(self, p, state):
        t0 = time.perf_counter()
        self.hs.run(p, state)
        return time.perf_counter() - t0


def cpu_baseline():
    """The reference's host FP64 solve (``HostSolve``): one whole config-1 solve (29 DGEMM
    products of 6144^3 with the O(d^2) work) timed on all host threads."""
    hs = HostSolve()
    hs.hs.run(0, {})  # warm the BLAS threads (one product, not timed)
    t, V, _ = hs.solve()
    assert V.shape == (NMAT, hs.d, NK)
    return {"value": round(NMAT * NK / t, 3), "unit": "quotes/s", "cores": hs.nth, "kind": "port",
            "cpu_model": hs.model,
            "sample": f"one whole FP64 solve of the SV lattice (U0 = I + dt L, {hs.niter} squarings, {NMAT - 1} "
                      f"chain products, payoff products; torch-CPU/MKL DGEMM, {hs.nth} threads, denormals "
                      f"flushed: {hs.ftz}) = {t:.2f} s; generator built once outside the timing"}


# ----------------------------------------------------------------------------------------
# Secondary workloads (not the headline line): config 0 (LV lattice), config 2 (Monte
# Carlo), and the squaring GEMM alone (the profiling case).

def _graph(step, dev, torch):
    """Capture one step (library launches only, no sync, no allocation) in a CUDA graph."""
    from oplib_b200.model import bind_stream
    s = torch.cuda.Stream(dev)
    s.wait_stream(torch.cuda.current_stream(dev))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        bind_stream(dev)
        g.capture_begin()
        step()
        g.capture_end()
    torch.cuda.current_stream(dev).wait_stream(s)
    bind_stream(dev)
    return g


def _time(fn, steps, stream, torch):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_lv(args):
    """Config 0: LV lattice n = 512, dt0 = 2^-14, 12 squarings, 7 chains, 8 quarterly
    maturities x 64 strikes = 512 quotes per solve; CUDA-graph replay of the solve."""
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import MODES, Lattice, bind_stream
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    lat = Lattice.local_vol(n=512, device=dev)
    plan = lat.plan(0.25, 2.0 ** -14)
    strikes = torch.tensor([0.5 + j / 63 for j in range(64)], dtype=torch.float64, device=dev)
    out = {}
    for mname in ["bf16x3", "fp32"]:
        mode = MODES[mname]
        ws = lat.workspace(64, mode)
        q = torch.empty(8, 64, dtype=torch.float64, device=dev)
        desc = lat.desc(plan, 0.25, 8, strikes)

        def step():
            _lib.call("opb_lattice_solve", C.byref(desc), mode, ws.data_ptr(), ws.numel(), q.data_ptr(), None)
        for _ in range(args.warmup):
            step()
        g = _graph(step, dev, torch)
        for _ in range(2):
            g.replay()
        ms = _time(g.replay, args.steps, stream, torch)
        out[mname] = {"ms_per_solve": round(ms, 4), "quotes_per_s": round(512 / (ms * 1e-3), 1)}
    line = {"metric": "priced quotes/sec, LV lattice n=512 (CUDA-graph replay)", "value": out["bf16x3"]["quotes_per_s"],
            "unit": "quotes/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": out["bf16x3"]["ms_per_solve"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic",
            "config": {"workload": "LV lattice 512 nodes, 12 squarings + 7 chains, 64 strikes x 8 maturities",
                       "niter": plan.niter}, "modes": out}
    return line


def run_mc(args):
    """Config 2: Monte Carlo on the LV(512) lattice, step kernel dt = 1/252 (7 squarings),
    2^20 paths x 504 steps, one MT19937 stream per path, barrier (0.7) and Asian calls.
    One step = step-kernel build + cumulative rows + guide table + the MC kernel.  The
    step kernel is squared in split-FP16 on the tensor cores with FP64 renormalisation
    (0.15 ms against 0.62 ms for the FP32 SIMT squaring, and closer to the FP64 kernel);
    the cumulative rows are FP32 as the configuration states."""
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import Lattice, bind_stream, cumulative_rows, guide_table, mc_run
    from oplib_b200.shard import allreduce_sums, path_range
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    lat = Lattice.local_vol(n=512, device=dev)
    plan = lat.plan(1 / 252, 2.0 ** -14)
    # weak scaling: 2^20 paths per GPU; runs past 623 steps use the state-array generator
    total_paths, nsteps = (1 << 20) * world, args.mc_steps
    path0, npaths = path_range(total_paths, rank, world)
    disc = math.exp(-0.03 * nsteps / 252)
    nblk = _lib.load().opb_mc_scratch_blocks(npaths)
    scratch = torch.empty(2 * nblk, dtype=torch.float64, device=dev)
    state = {}

    def prep():
        P = lat.kernel(1 / 252, 2.0 ** -14, mode="fp16x3", plan=plan)
        Cm = cumulative_rows(P)
        state["C"], state["g"] = Cm, guide_table(Cm)

    graph = []

    def step(with_kernel=True):
        if with_kernel:
            if graph:
                graph[0].replay()
            else:
                prep()
        sums, _ = mc_run(state["C"], lat.y0, nsteps, 5489, npaths, path0=path0, guide=state["g"], x=lat.x,
                         disc=disc, scratch=scratch)
        state["sums"] = allreduce_sums(sums)

    for _ in range(args.warmup):
        step()
    # the step-kernel build, cumulative rows and guide table (about 20 short launches) as one
    # CUDA graph; its buffers stay valid across replays
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        prep()
    bind_stream(dev)
    graph.append(g)
    step()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    ms = _time(step, args.steps, stream, torch)
    ms_mc = _time(lambda: step(False), args.steps, stream, torch)
    if world > 1:
        t = torch.tensor([ms, ms_mc], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_mc = float(t[0]), float(t[1])
    # the same kernel writing every int16 state (the reference's y_sk output): 2 bytes per
    # path-step to HBM, 1.06 GB for 2^20 x 504 -- its achieved write bandwidth
    ypaths = torch.empty(nsteps, npaths, dtype=torch.int16, device=dev)

    def step_paths():
        _lib.call("opb_mc_mt19937", state["C"].data_ptr(), lat.d, 1, state["g"].data_ptr(), state["g"].shape[1],
                  lat.d, lat.y0,
                  nsteps, 5489, path0, npaths, ypaths.data_ptr(), None, 1.0, 0.7, 1.0, None, None)

    step_paths()
    ms_paths = _time(step_paths, args.steps, stream, torch)
    del ypaths
    hbm, _, _, src = _peaks()
    gbs = 2.0 * npaths * nsteps / (ms_paths * 1e-3) / 1e9
    sums = state["sums"].cpu().numpy() / total_paths
    samples = total_paths * nsteps
    line = {"metric": "Monte Carlo path-steps/sec (MT19937 per path, inverse-CDF on FP32 cumulative rows)",
            "value": round(samples / (ms * 1e-3), 1), "unit": "path-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32 RNG + f32 compare", "data": "synthetic",
            "config": {"workload": f"LV(512) lattice, dt=1/252 step kernel, 2^20 paths per GPU x {nsteps} steps, "
                                   "barrier 0.7 + Asian, K=1", "paths": total_paths, "steps_per_path": nsteps,
                       "generator": "register cursors" if nsteps <= 623 else "624-word state in local memory",
                       "parallelism": f"path ranges x{world}, one all-reduce of 2 sums",
                       "step": "step-kernel build + cumulative rows + guide table (one CUDA graph) + MC kernel"},
            "mc_kernel_only": {"ms": round(ms_mc, 3), "path_steps_per_s": round(samples / (ms_mc * 1e-3), 1)},
            "with_state_output": {"ms": round(ms_paths, 3), "path_steps_per_s":
                                  round(npaths * nsteps / (ms_paths * 1e-3), 1), "hbm_write_GB_s": round(gbs, 1),
                                  "frac_of_hbm": round(gbs / hbm, 4), "peak_source": src},
            "prices": {"barrier_do_call": float(sums[0]), "asian_call": float(sums[1])}}
    if args.cpu and rank == 0:
        from oracle import oracle_c as OC
        nth = os.cpu_count() or 1
        Cm = state["C"].cpu().numpy()
        xs = lat.x.cpu().numpy()
        n_cpu = 1 << 15
        t0 = time.perf_counter()
        OC.mc_paths(Cm, lat.y0, 5489, 0, n_cpu, nsteps, x=xs, disc=disc, want_paths=False, nthreads=nth)
        tc = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": round(n_cpu * nsteps / tc, 1), "unit": "path-steps/s", "cores": nth,
                                "kind": "port", "sample": f"{n_cpu} paths x {nsteps} steps, C oracle, {nth} threads"}
    return line


def _fp64_lv_quotes(lat, plan, strikes, nmat, period, torch):
    """FP64 solve of one ELL lattice on the device with torch (accuracy reference)."""
    d = lat.d
    cols = lat.cols.view(d, -1).long()
    vals = lat.vals.view(d, -1)
    L = torch.zeros(d, d, dtype=torch.float64, device=lat.device)
    mask = cols >= 0
    rows = torch.arange(d, device=lat.device).unsqueeze(1).expand_as(cols)
    L.index_put_((rows[mask], cols[mask]), vals[mask], accumulate=True)
    P = torch.eye(d, dtype=torch.float64, device=lat.device) + plan.dt * L
    for _ in range(plan.niter):
        P = P @ P
        P /= P.sum(dim=1, keepdim=True)
    K = torch.tensor(strikes, dtype=torch.float64, device=lat.device)
    G = torch.clamp(lat.x.unsqueeze(1) - K.unsqueeze(0), min=0.0)
    out, Pm = [], P
    for m in range(1, nmat + 1):
        if m > 1:
            Pm = Pm @ P
            Pm /= Pm.sum(dim=1, keepdim=True)
        out.append(math.exp(-lat.rate * period * m) * (Pm[lat.y0] @ G))
    return torch.stack(out)


def run_calibrate(args):
    """Calibration loop: --nlat local-vol problems (n = 512, 8 quarterly maturities x 32
    strikes = 256 quotes each) fitted for (level, skew, width) by Levenberg-Marquardt from
    two starts; each iteration rebuilds 7 generators per problem and start on the device
    (central differences) and prices all of them in one batched execute.  Targets are the
    device's own prices at seeded parameters, so the recovered parameters measure the
    loop; a step is one full calibration of all problems."""
    import time
    import numpy as np
    import torch
    from oplib_b200.calibrate import LVBatchPricer, best_of_starts, lm_calibrate, multistart
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    M = args.nlat
    rng = np.random.default_rng(20261)
    rates = rng.uniform(0.0, 0.05, M)
    truth = np.stack([rng.uniform(0.12, 0.4, M), rng.uniform(-0.25, 0.25, M), rng.uniform(0.3, 1.0, M)], axis=1)
    strikes = np.linspace(0.6, 1.5, 32)
    t0 = time.perf_counter()
    pricer = LVBatchPricer([512] * (2 * M), np.concatenate([rates, rates]), strikes, 8, 0.25, device=dev)
    plan_s = time.perf_counter() - t0
    targets = pricer.quotes(np.concatenate([truth, truth]))[:M]
    tg, theta0 = multistart(targets)
    out = None
    for _ in range(args.warmup):
        lm_calibrate(pricer, tg, theta0, iters=3)
    torch.cuda.synchronize()
    calls0 = pricer.calls
    t0 = time.perf_counter()
    iters = []
    for _ in range(args.steps):
        out = lm_calibrate(pricer, tg, theta0, iters=40, ftol=5e-8)
        iters.append(out["iterations"])
    torch.cuda.synchronize()
    sec = (time.perf_counter() - t0) / args.steps
    ncalls = (pricer.calls - calls0) / args.steps
    theta, rms = best_of_starts(out, M)
    return {"metric": "local-vol calibrations/sec (3 parameters to 256 lattice quotes, on-device pricing)",
            "value": round(M / sec, 2), "unit": "calibrations/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp16x3 lattice, fp64 host solve", "data": "synthetic",
            "config": {"workload": f"{M} LV problems, n=512, 8 x 32 quotes, 2 starts x 7 lattices per iteration",
                       "lattices_per_iteration": 14 * M},
            "iterations": int(max(iters)), "pricer_calls_per_step": ncalls,
            "ms_per_iteration": round(sec * 1e3 / ncalls, 2),
            # the quotes pin the prices, not always the parameters (a narrow or far bump of
            # small skew changes the 256 prices by less than the pricer's noise): the fit is
            # judged by its price residual; the parameter recovery is reported beside it
            "max_rms_price_residual": float(rms.max()), "median_rms_price_residual": float(np.median(rms)),
            "recovered_within_1e-3": float(np.mean(np.all(np.abs(theta - truth) < 1e-3, axis=1))),
            "median_param_err": float(np.median(np.abs(theta - truth).max(axis=1))),
            "plan_seconds": round(plan_s, 2)}


def run_batch(args):
    """Config 3: calibration sweep of 512 seeded local-vol lattices, n uniform over
    {256, 384, ..., 2048}, 32 strikes x 8 quarterly maturities each (131,072 quotes);
    all lattices' squarings of a level in one persistent launch, the whole sweep replayed
    from a CUDA graph; autotuned tile shape / work order."""
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import Batch, bind_stream, calibration_sweep
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    nlat = args.nlat
    lats, params = calibration_sweep(nlat=nlat, device=dev)
    strikes = [0.5 + j / 31.0 for j in range(32)]
    nquotes = nlat * 8 * 32
    order = None
    res = {}
    for mname in ["fp16x3", "bf16x3"]:
        t0 = time.perf_counter()
        b = Batch(lats, strikes, 8, 0.25, 2.0 ** -14, mode=mname, autotune=True)
        torch.cuda.synchronize()
        t_plan = time.perf_counter() - t0
        q = torch.empty(nlat, 8, 32, dtype=torch.float64, device=dev)
        for _ in range(args.warmup):
            b.execute(q)
        g = _graph(lambda: b.execute(q), dev, torch)
        g.replay()
        ms = _time(g.replay, args.steps, stream, torch)
        if order is None:
            order = sorted(range(nlat), key=lambda i: -b.plans[i].niter)
            sample = order[:8] + order[-4:]
            refs = {i: _fp64_lv_quotes(lats[i], b.plans[i], strikes, 8, 0.25, torch) for i in sample}
        errs = {int(i): float((q[i] - refs[i]).abs().max().item()) for i in sample}
        # whole-sweep time of every configuration (the autotuner picks on level 0 alone)
        sweep_ms = []
        berm = None
        if mname == "fp16x3":
            # Bermudan puts on every lattice (32 strikes, 8 quarterly exercise dates) by
            # backward induction on the same plan: squarings plus 8 batched induction products
            qb = torch.empty(nlat, 32, dtype=torch.float64, device=dev)
            b.execute_bermudan(put=True, exercise=True, quotes=qb)
            ms_b = _time(lambda: b.execute_bermudan(put=True, exercise=True, quotes=qb), max(2, args.steps), stream,
                         torch)
            berm = {"quotes_per_s": round(nlat * 32 / (ms_b * 1e-3), 1), "ms_per_sweep": round(ms_b, 3),
                    "quotes_per_sweep": nlat * 32}
            chosen = b.config
            for cfg in range(_lib.load().opb_batch_num_configs()):
                b.set_config(cfg)
                b.execute(q)
                sweep_ms.append(round(_time(lambda: b.execute(q), 2, stream, torch), 2))
            b.set_config(chosen)
        res[mname] = dict(ms=ms, plan_s=t_plan, tune=b.tune_ms, cfg=b.config, launches=b.launches(), errs=errs,
                          q=q, plans=b.plans, sweep_ms=sweep_ms, berm=berm)
        del g, b
    prim = res["fp16x3"]
    ms = prim["ms"]
    useful = sum(2.0 * p["n"] ** 3 * (pl.niter + 7) for p, pl in zip(params, prim["plans"]))
    line = {"metric": "priced quotes/sec, batched calibration sweep (split tensor-core products, one launch per level)",
            "value": round(nquotes / (ms * 1e-3), 1), "unit": "quotes/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp16x3", "data": "synthetic",
            "config": {"workload": f"{nlat} LV lattices, n in 256..2048 step 128 (seed 20260), 32 strikes x 8 "
                                   "maturities, CUDA-graph replay", "nlat": nlat,
                       "niter_range": [min(p.niter for p in prim["plans"]), max(p.niter for p in prim["plans"])]},
            "useful_tflops": round(useful / (ms * 1e-3) / 1e12, 1),
            "mma_tflops": round(3 * useful / (ms * 1e-3) / 1e12, 1),
            "autotune_ms_chain_product": [round(x, 3) for x in prim["tune"]], "config_chosen": prim["cfg"],
            "sweep_ms_per_config": prim["sweep_ms"],
            "launches_per_sweep": prim["launches"], "plan_seconds": round(prim["plan_s"], 2),
            "max_abs_err_vs_fp64_sample": max(prim["errs"].values()), "sample_errs": prim["errs"],
            "bf16x3": {"quotes_per_s": round(nquotes / (res["bf16x3"]["ms"] * 1e-3), 1),
                       "max_abs_err_vs_fp64_sample": max(res["bf16x3"]["errs"].values())},
            "bermudan_puts_fp16x3": prim["berm"]}
    q = prim["q"]
    b = type("P", (), {"plans": prim["plans"]})
    if args.compare:
        b32 = Batch(lats, strikes, 8, 0.25, 2.0 ** -14, mode="fp32", autotune=False)
        q32 = b32.execute()
        torch.cuda.synchronize()
        ms32 = _time(lambda: b32.execute(q32), 1, stream, torch)
        line["fp32_quotes_per_s"] = round(nquotes / (ms32 * 1e-3), 1)
        line["speedup_vs_fp32"] = round(ms32 / ms, 2)
        line["max_abs_diff_vs_fp32"] = float((q - q32).abs().max().item())
        line["fp32_max_abs_err_vs_fp64_sample"] = max(
            float((q32[i] - _fp64_lv_quotes(lats[i], b.plans[i], strikes, 8, 0.25, torch)).abs().max().item())
            for i in sample)
    return line


def run_batch_sharded(args):
    """Config 3 across the ranks of a torchrun job: the 512 seeded lattices are bin-packed by
    n^3 (longest processing time first), each rank plans, autotunes and solves its own set,
    and one all-gather gives every rank all quotes.  A step is the local sweep plus the
    gather; the time is the max over ranks, the value all quotes over that time."""
    import torch
    import torch.distributed as dist
    from oplib_b200.model import Batch, Lattice, bind_stream, calibration_sweep
    from oplib_b200.shard import gather_quotes, lpt_partition
    world, rank = dist.get_world_size(), dist.get_rank()
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    nlat = args.nlat
    _, params = calibration_sweep(nlat=nlat, device=dev, build=False)
    bins = lpt_partition([float(p["n"]) ** 3 for p in params], world)
    mine = bins[rank]
    strikes = [0.5 + j / 31.0 for j in range(32)]
    lats = [Lattice.local_vol(device=dev, **params[i]) for i in mine]
    b = Batch(lats, strikes, 8, 0.25, 2.0 ** -14, mode="fp16x3", autotune=True)
    q = torch.empty(len(mine), 8, 32, dtype=torch.float64, device=dev)
    out = {}

    def step():
        b.execute(q)
        out["q"] = gather_quotes(q, bins, nlat)

    for _ in range(args.warmup):
        step()
    dist.barrier()
    ms = _time(step, args.steps, stream, torch)
    t = torch.tensor([ms], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    # every rank holds all quotes: rank 0 checks two lattices of the last rank against FP64
    errs = {}
    if rank == 0:
        for i in bins[-1][:2]:
            lat = Lattice.local_vol(device=dev, **params[i])
            plan = lat.plan(0.25, 2.0 ** -14)
            errs[int(i)] = float((out["q"][i] - _fp64_lv_quotes(lat, plan, strikes, 8, 0.25, torch)).abs().max().item())
    nq = nlat * 8 * 32
    return {"metric": "priced quotes/sec, batched calibration sweep sharded over ranks (LPT bins, one all-gather)",
            "value": round(nq / (ms * 1e-3), 1), "unit": "quotes/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "fp16x3", "data": "synthetic",
            "config": {"workload": f"{nlat} LV lattices, n in 256..2048 step 128 (seed 20260), 32 strikes x 8 "
                                   "maturities", "parallelism": f"lattice bins x{world}",
                       "lattices_per_rank": [len(x) for x in bins]},
            "max_abs_err_vs_fp64_sample": max(errs.values()) if errs else None}


def _surrogate_inference_only(args, dev, stream, torch):
    """--epochs 0: inference timing alone (randomly initialised members, no data, no
    training) on 2^20 seeded feature vectors -- the kernel-profiling case."""
    from oplib_b200 import _lib
    from oplib_b200.surrogate import RANGES, Surrogate
    sur = Surrogate(members=args.members, device=dev)
    for m in range(sur.members):
        _lib.call("opb_mlp_pack", sur.theta[m].data_ptr(), sur.packed[m * sur.stride:].data_ptr())
    n = 1 << 20
    rng = np.random.default_rng(0)
    feat = torch.from_numpy(np.column_stack([rng.uniform(lo, hi, n) for lo, hi in RANGES])).to(dev)
    base = torch.zeros(n, dtype=torch.float64, device=dev)
    ws = torch.empty(int(sur.lib.opb_mlp_infer_workspace_bytes(n, sur.members)), dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        sur.predict(feat, base, ws)
    ms = _time(lambda: sur.predict(feat, base, ws), args.steps, stream, torch)
    return {"metric": "surrogate quotes/sec (ensemble MLP on tensor cores), inference only", "value":
            round(n / (ms * 1e-3), 1), "unit": "quotes/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 weights/activations, fp32 accumulate", "data": "synthetic (random weights)",
            "config": {"workload": f"2^20 quotes, ensemble of {sur.members} MLPs 8-256x4-1, untrained"}}


def run_surrogate(args):
    """Config 4: ensemble of MLP surrogates (8 -> 256 x 4 -> 1, GELU) trained by the
    library's kernels on ~2^21 quotes that the batched lattice solver generates (local-vol
    lattices, n = 1024), then inference on 2^20 held-out quotes on the tensor cores;
    quotes whose ensemble spread exceeds 5 bp fall back to the lattice.  Reports surrogate
    quotes/s, the lattice's quotes/s for the same family, fallback rate and errors
    against the lattice."""
    import torch
    from oplib_b200.model import Batch, bind_stream
    from oplib_b200.surrogate import NMAT, PERIOD, LM, Surrogate, lattice_quotes
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    if args.epochs == 0:
        return _surrogate_inference_only(args, dev, stream, torch)
    t0 = time.perf_counter()
    train = lattice_quotes(args.train_lattices, seed=2026, device=dev)
    test = lattice_quotes(1024, seed=31337, device=dev)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    sur = Surrogate(members=args.members, device=dev)
    sur.train(train, epochs=args.epochs, batch=4096, lr=2e-3)
    n = 1 << 20
    reps = (n + test.feat.shape[0] - 1) // test.feat.shape[0]
    feat = test.feat.repeat(reps, 1)[:n].contiguous()
    base = test.base.repeat(reps)[:n].contiguous()
    ws = torch.empty(int(sur.lib.opb_mlp_infer_workspace_bytes(n, sur.members)), dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        sur.predict(feat, base, ws)
    ms_inf = _time(lambda: sur.predict(feat, base, ws), args.steps, stream, torch)
    # accuracy on the held-out quotes
    iv, spread = sur.predict(test.feat, test.base, ws)
    err = (iv - test.iv).abs() * 1e4
    errb = (test.base - test.iv).abs() * 1e4
    fb = spread * 1e4 > 5.0
    acc = ~fb
    fb_lat = torch.unique(test.lattice[fb]).numel()
    # lattice throughput for the same family (one 512-lattice sweep of the test distribution)
    from oplib_b200.model import Lattice
    rng = np.random.default_rng(7)
    lats = [Lattice.local_vol(n=1024, level=float(rng.uniform(0.1, 0.4)), skew=float(rng.uniform(-0.3, 0.3)),
                              width=float(rng.uniform(0.2, 1.0)), rate=float(rng.uniform(0.0, 0.05)), floor=0.01,
                              device=dev) for _ in range(512)]
    bt = Batch(lats, np.exp(LM), NMAT, PERIOD, 2.0 ** -14, mode="fp16x3", autotune=True)
    qq = bt.execute()
    g = _graph(lambda: bt.execute(qq), dev, torch)
    g.replay()
    ms_lat = _time(g.replay, 3, stream, torch)
    lat_qps = 512 * NMAT * 64 / (ms_lat * 1e-3)
    sur_qps = n / (ms_inf * 1e-3)
    # effective: surrogate for accepted quotes, lattice re-solve of every lattice holding a fallback
    n_test = test.feat.shape[0]
    eff_s = ms_inf * 1e-3 * n_test / n + (fb_lat / 512) * ms_lat * 1e-3
    # a 2-member operating point (the first two members): half the inference work, the
    # spread of a pair as the fallback test
    ms2 = _time(lambda: sur.predict(feat, base, ws, members=2), args.steps, stream, torch)
    iv2, sp2 = sur.predict(test.feat, test.base, ws, members=2)
    err2 = (iv2 - test.iv).abs() * 1e4
    acc2 = sp2 * 1e4 <= 5.0
    two = {"quotes_per_s": round(n / (ms2 * 1e-3), 1), "ms": round(ms2, 3),
           "speedup_vs_lattice": round(n / (ms2 * 1e-3) / (512 * NMAT * 64 / (ms_lat * 1e-3)), 1),
           "fallback_rate": round(float((~acc2).float().mean().item()), 4),
           "accepted_err_bp": {"rms": round(float(err2[acc2].pow(2).mean().sqrt().item()), 2),
                               "p99": round(float(torch.quantile(err2[acc2].float(), 0.99).item()), 2)},
           "all_err_bp": {"rms": round(float(err2.pow(2).mean().sqrt().item()), 2)}}
    q = lambda x, p: float(torch.quantile(x.float(), p).item()) if x.numel() else float("nan")
    return {"metric": "surrogate quotes/sec (ensemble MLP on tensor cores) vs lattice quotes/sec",
            "value": round(sur_qps, 1), "unit": "quotes/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_inf, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 weights/activations, fp32 accumulate", "data": "synthetic (lattice-generated)",
            "config": {"workload": f"2^20 quotes, ensemble of {sur.members} MLPs 8-256x4-1, trained on "
                                   f"{train.feat.shape[0]} quotes from {args.train_lattices} lattices, "
                                   f"{args.epochs} epochs, batch 4096", "members": sur.members},
            "lattice_quotes_per_s": round(lat_qps, 1), "speedup_vs_lattice": round(sur_qps / lat_qps, 1),
            "fallback_rate": round(float(fb.float().mean().item()), 4),
            "fallback_lattices": int(fb_lat), "test_quotes": int(n_test),
            "accepted_err_bp": {"rms": round(float(err[acc].pow(2).mean().sqrt().item()), 2) if acc.any() else None,
                                "p99": round(q(err[acc], 0.99), 2), "max": round(float(err[acc].max().item()), 2)
                                if acc.any() else None},
            "all_err_bp": {"rms": round(float(err.pow(2).mean().sqrt().item()), 2), "p99": round(q(err, 0.99), 2)},
            "baseline_err_bp": {"rms": round(float(errb.pow(2).mean().sqrt().item()), 2), "p99": round(q(errb, 0.99), 2)},
            "effective_quotes_per_s_with_fallback": round(n_test / eff_s, 1),
            "spread_threshold_bp": 5.0, "two_members": two,
            "train_seconds": round(sur.train_seconds, 1), "data_seconds": round(t_data, 1),
            "final_train_mse": sur.history[-1][2]}


def run_renorm(args):
    """The FP64 row renormalisation + split kernel alone at size d (E-form with both
    splits): algorithmic traffic 16 bytes per element (read 4, write 4 + 4 x 2) + the
    row-sum partials."""
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import bind_stream
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    d = args.d
    X = torch.empty(d, d, dtype=torch.float32, device=dev).uniform_(0, 1e-3)
    np_ = d // 128
    part = torch.empty(np_ * d, dtype=torch.float64, device=dev).uniform_(0, 1e-3)
    A = [torch.empty(d, d, dtype=torch.bfloat16, device=dev) for _ in range(4)]
    f = lambda: _lib.call("opb_renorm_rows", d, X.data_ptr(), part.data_ptr(), np_, 0, *[a.data_ptr() for a in A], 0)
    for _ in range(args.warmup):
        f()
    ms = _time(f, args.steps, torch.cuda.current_stream(dev), torch)
    hbm, _, _, src = _peaks()
    byts = 16.0 * d * d + 8.0 * np_ * d
    gbs = byts / (ms * 1e-3) / 1e9
    return {"metric": "FP64 renormalisation + split, achieved GB/s", "value": round(gbs, 1), "unit": "GB/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 -> bf16",
            "data": "synthetic", "config": {"workload": f"k_renorm64 E-form with A and B splits, d={d}"},
            "frac_of_peak": round(gbs / hbm, 4), "peak_source": src}


def run_gemv(args):
    """Backward-induction GEMV of the drop-in entry points on a d x d column-major FP32
    matrix (the reference's layout; 151 MB at d = 6144, larger than L2): opcuda_sgemvT
    (warp per column: the warp-per-row GEMV of a source-major kernel) and opcuda_sgemv
    (column chunks + ordered reduction).  Algorithmic bytes: 4 d^2 + 12 d per call."""
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import bind_stream
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    d = args.d
    A = torch.empty(d * d, dtype=torch.float32, device=dev).uniform_(0, 1.0 / d)
    x = torch.empty(d, dtype=torch.float32, device=dev).uniform_()
    y = torch.zeros(d, dtype=torch.float32, device=dev)
    hbm, _, _, src = _peaks()
    byts = 4.0 * d * d + 12.0 * d
    res = {}
    for name in ("opcuda_sgemvT", "opcuda_sgemv"):
        f = lambda: _lib.call(name, d, d, 1.0, A.data_ptr(), d, x.data_ptr(), 1, 0.0, y.data_ptr(), 1)
        for _ in range(max(3, args.warmup)):
            f()
        ms = _time(f, args.steps, stream, torch)
        res[name] = {"ms": round(ms, 4), "GB_s": round(byts / (ms * 1e-3) / 1e9, 1),
                     "frac": round(byts / (ms * 1e-3) / 1e9 / hbm, 4)}
    v = res["opcuda_sgemvT"]
    return {"metric": "backward-induction GEMV achieved GB/s (warp-per-row, source-major kernel)", "value": v["GB_s"],
            "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": v["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"GEMV on a {d} x {d} FP32 matrix ({4 * d * d / 1e6:.0f} MB > L2)"},
            "roofline": {"bound": "hbm", "achieved": v["GB_s"], "peak": hbm, "unit": "GB/s", "frac": v["frac"],
                         "peak_source": src},
            "column_major_N": res["opcuda_sgemv"]}


# OPBench figures published by the reference for its first box (Tesla "1060" GPU0 and its
# host), docs/benchmarks/nehalem-tesla1060.jpg; context only (2009-era hardware).
OPBENCH_PUBLISHED = {
    "sgemm_576x100": (340.0, "GF/s"), "sgemm4_40x576": (368.6, "GF/s"), "sgemv_576x100": (2.5, "GF/s"),
    "mt_uniforms": (1470.5, "M/s"), "mt_uniforms_with_copy": (510.5, "M/s"), "lv_kernels": (108.5, "GF/s"),
    "lv_mc": (142.9, "M eval/s"), "sv_kernels": (256.5, "GF/s"), "sv_mc": (41.2, "M eval/s"),
    "cpu_sgemm": (35.2, "GF/s"), "cpu_dgemm": (31.0, "GF/s"), "cpu_mt": (724.1, "M/s"), "cpu_lv_mc": (560.2, "M eval/s"),
    "cpu_sv_mc": (485.5, "M eval/s"),
}


def run_refbench(args):
    """The reference's own benchmark workloads (benchmarks/opbench/CBenchmarks.cs and the
    benchmarks/*/Program.cs drivers) on this GPU through the drop-in entry points, and their
    CPU counterparts on this host's cores in the same run:
      SGEMM 576^3 x 100 (opcuda_sgemm), grouped SGEMM4 40 x 576^3 (opcuda_sgemm4 task table),
      SGEMV 576 x 100 (opcuda_sgemv), MT uniforms 20 batches of 102,400 with and without the
      copy to the host (opcuda_mt_benchmark), LV (128 states, sigma 0.25, r 0.05) and SV (64 x 8
      states) step kernels for 7-day steps by squaring (GF/s = 2 d^3 per product / time) and
      their Monte Carlo (opcuda_mc1f, 40 weekly steps; LV 20 x 102,400 paths, SV 4,096 paths;
      M eval/s = path-steps / wall time including the per-batch copy of the int16 states, as
      the reference times them); CPU: csgemm / cdgemm (torch-CPU), cmt (C MT19937 restatement,
      all threads), clv / csv Monte Carlo (C restatement, all threads; 102,400 x 120 and
      102,400 x 100 paths x 40 steps) on the same step kernels."""
    import platform
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import Lattice, bind_stream, cumulative_rows
    from oracle import oracle_c as OC
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    lib = _lib.load()
    res = {}
    ncpu = os.cpu_count() or 1

    def put(name, value, unit, **kw):
        pub = OPBENCH_PUBLISHED.get(name)
        res[name] = dict(value=round(value, 2), unit=unit, **kw)
        if pub:
            res[name]["published_reference"] = pub[0]

    # ---- SGEMM 576^3 x 100 (column-major drop-in, FP32 SIMT)
    d = 576
    A = torch.empty(d * d, device=dev).uniform_()
    B = torch.empty(d * d, device=dev).uniform_()
    Cc = torch.empty(d * d, device=dev)
    f = lambda: lib.opcuda_sgemm(d, d, d, 1.0, A.data_ptr(), d, B.data_ptr(), d, 0.0, Cc.data_ptr(), d)
    f()
    ms = _time(f, 100, stream, torch)
    put("sgemm_576x100", 2.0 * d ** 3 / (ms * 1e-3) / 1e9, "GF/s")
    # ---- grouped SGEMM4: 40 products of 576^3 through one task table (64 x 16 C tiles)
    mats = [(torch.empty(d * d, device=dev).uniform_(), torch.empty(d * d, device=dev).uniform_(),
             torch.empty(d * d, device=dev)) for _ in range(40)]
    sz = lib.opb_sgemm4_task_size()
    tasks = []
    for i, (a_, b_, c_) in enumerate(mats):
        for bx in range(d // 64):
            for by in range(d // 16):
                tasks.append((i, bx, by, d, d, d, a_.data_ptr(), b_.data_ptr(), c_.data_ptr()))
    rec = np.zeros((len(tasks), sz // 8), dtype=np.int64)
    for t, (i, bx, by, m, n, k, a_, b_, c_) in enumerate(tasks):
        rec[t, :3] = np.array([i, bx, by, m, n, k], dtype=np.int32).view(np.int64)
        rec[t, 3:6] = [a_, b_, c_]
    drec = torch.from_numpy(rec.ravel()).to(dev)
    ptrs = torch.tensor([drec.data_ptr() + t * sz for t in range(len(tasks))], dtype=torch.int64, device=dev)
    f = lambda: lib.opcuda_sgemm4(len(tasks), ptrs.data_ptr())
    f()
    ms = _time(f, 5, stream, torch)
    put("sgemm4_40x576", 40 * 2.0 * d ** 3 / (ms * 1e-3) / 1e9, "GF/s")
    del mats, drec, ptrs
    # ---- SGEMV 576 x 100
    x = torch.empty(d, device=dev).uniform_()
    y = torch.empty(d, device=dev)
    f = lambda: lib.opcuda_sgemv(d, d, 1.0, A.data_ptr(), d, x.data_ptr(), 1, 0.0, y.data_ptr(), 1)
    f()
    ms = _time(f, 100, stream, torch)
    put("sgemv_576x100", 2.0 * d * d / (ms * 1e-3) / 1e9, "GF/s")
    # ---- MT uniforms: 20 batches of 102,400 (25 per stream, 4096 streams)
    nb, ns = 20, 4096 * 25
    mt = torch.zeros(lib.opcuda_mc_status_sz(), dtype=torch.int32, device=dev)
    seed = np.random.default_rng(5489).integers(0, 2**31 - 1, lib.opcuda_mc_nrng()).astype(np.uint32)
    assert lib.opcuda_mc_setseed(seed.ctypes.data, mt.data_ptr()) == 0
    unif = torch.empty(ns, device=dev)
    host = torch.empty(ns, dtype=torch.float32).pin_memory()
    lib.opcuda_mt_benchmark(mt.data_ptr(), unif.data_ptr(), ns)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(nb):
        lib.opcuda_mt_benchmark(mt.data_ptr(), unif.data_ptr(), ns)
    torch.cuda.synchronize()
    put("mt_uniforms", nb * ns / (time.perf_counter() - t0) / 1e6, "M/s")
    t0 = time.perf_counter()
    for _ in range(nb):
        lib.opcuda_mt_benchmark(mt.data_ptr(), unif.data_ptr(), ns)
        host.copy_(unif)
    torch.cuda.synchronize()
    put("mt_uniforms_with_copy", nb * ns / (time.perf_counter() - t0) / 1e6, "M/s")

    # ---- LV and SV: 7-day step kernels by squaring, then Monte Carlo over 40 weekly steps
    step, day = 7.0 / 365.25, 1.0 / 365.25
    cpu_rows = {}
    for name, lat, nbatch, nscen in [("lv", Lattice.local_vol(n=128, level=0.25, skew=0.0, width=1.0, rate=0.05,
                                                                device=dev), 20, 4096 * 25),
                                     ("sv", Lattice.stoch_vol(nx=64, nv=8, rate=0.05, device=dev), 1, 4096)]:
        plan = lat.plan(step, day)
        dd = lat.d
        P = lat.kernel(step, day, mode="fp32", plan=plan)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(10):
            P = lat.kernel(step, day, mode="fp32", plan=plan)
        torch.cuda.synchronize()
        sec = (time.perf_counter() - t0) / 10
        put(f"{name}_kernels", 2.0 * dd ** 3 * plan.niter / sec / 1e9, "GF/s", d=dd, niter=plan.niter)
        Cm = cumulative_rows(P)
        Ccm = Cm.t().contiguous()  # the reference's column-major layout
        mk = torch.zeros(40, dtype=torch.int32, device=dev)
        ysk = torch.empty(nscen * 40, dtype=torch.int16, device=dev)
        yh = torch.empty(nscen * 40, dtype=torch.int16).pin_memory()
        assert lib.opcuda_mc_setseed(seed.ctypes.data, mt.data_ptr()) == 0
        lib.opcuda_mc1f(mt.data_ptr(), lat.y0, ysk.data_ptr(), nscen, 40, dd, Ccm.data_ptr(), mk.data_ptr(),
                        yh.data_ptr())
        t0 = time.perf_counter()
        for _ in range(nbatch):
            assert lib.opcuda_mc1f(mt.data_ptr(), lat.y0, ysk.data_ptr(), nscen, 40, dd, Ccm.data_ptr(),
                                   mk.data_ptr(), yh.data_ptr()) == 0
        sec = time.perf_counter() - t0
        put(f"{name}_mc", 40.0 * nbatch * nscen / sec / 1e6, "M eval/s", paths=nbatch * nscen, steps=40,
            includes="copy of the int16 states to the host per batch")
        cpu_rows[name] = (Cm.cpu().numpy(), lat.y0, dd, P.double().cpu(), plan)

    # ---- CPU counterparts on this host's cores
    for dt, name in [(torch.float32, "cpu_sgemm"), (torch.float64, "cpu_dgemm")]:
        a_ = torch.rand(d, d, dtype=dt)
        torch.mm(a_, a_)
        t0 = time.perf_counter()
        for _ in range(100):
            torch.mm(a_, a_)
        put(name, 100 * 2.0 * d ** 3 / (time.perf_counter() - t0) / 1e9, "GF/s", threads=torch.get_num_threads())
    lo = OC.load()
    per = (4096 * 25) // ncpu
    t0 = time.perf_counter()
    lo.oracle_mt_benchmark(per, 2000, ncpu, 5489)
    put("cpu_mt", ncpu * per * 2000 / (time.perf_counter() - t0) / 1e6, "M/s", threads=ncpu,
        note="MT19937 (the reference's CPU path used MKL MT2203)")
    for name, npaths in [("lv", 4096 * 25 * 120), ("sv", 4096 * 25 * 100)]:
        Cm, y0, dd, _, _ = cpu_rows[name]
        t0 = time.perf_counter()
        OC.mc_paths(Cm, y0, 5489, 0, npaths, 40, want_paths=False, nthreads=ncpu)
        put(f"cpu_{name}_mc", 40.0 * npaths / (time.perf_counter() - t0) / 1e6, "M eval/s", threads=ncpu,
            paths=npaths, steps=40)
    lvmc = res["lv_mc"]["value"]
    return {"metric": "reference benchmark suite (OPBench workloads): LV Monte Carlo M eval/s headline",
            "value": lvmc, "unit": "M eval/s", "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": round(lvmc / OPBENCH_PUBLISHED["lv_mc"][0], 1),
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "OPBench workloads (CBenchmarks.cs), drop-in entry points"},
            "host": {"cpu": platform.processor() or platform.machine(), "nproc": ncpu},
            "results": res,
            "note": "published_reference = the reference's own OPBench figure on a 2009 Tesla box (context)"}


def run_bermudan(args):
    """Bermudan puts on the SV lattice of the headline (d = 6144, 128 strikes, exercisable
    every 0.25 y to 4 y) by backward induction on the period kernel: 14 split squarings,
    then 16 induction products P1 . V (6144 x 6144 x 128) with the FP64 exercise step.  Two
    plain-FP32 arms: the library's SIMT path (`opb_lattice_bermudan` in OPB_FP32_RENORM) and
    cuBLAS SGEMM (TF32 off) with the same FP64 row renormalisation and FP64 step, the
    faster one being `speedup_vs_fp32`; the FP64 reference does everything in FP64 with
    torch on the device."""
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import MODES, Lattice, bind_stream
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    lat = Lattice.stoch_vol(**SV, device=dev)
    plan = lat.plan(PERIOD, DT0)
    strikes = torch.tensor(STRIKES, dtype=torch.float64, device=dev)
    desc = lat.desc(plan, PERIOD, NMAT, strikes)
    disc = math.exp(-lat.rate * PERIOD)
    x = lat.x
    ex = torch.clamp(strikes.unsqueeze(0) - x.unsqueeze(1), min=0.0)  # put exercise values [d, nK]

    def induction(P1, dtype):
        V = ex.clone()
        for m in range(NMAT - 1, -1, -1):
            V = disc * (P1 @ V.to(dtype)).double()
            if m >= 1:
                V = torch.maximum(V, ex)
        return V[lat.y0]

    out = {}
    for mode in ("bf16x3", "fp16x3", "fp32"):  # fp32: the library's SIMT path with FP64 renormalisation
        md = MODES[mode]
        ws = lat.workspace(NK, md)
        q = torch.empty(NK, dtype=torch.float64, device=dev)
        f = lambda: _lib.call("opb_lattice_bermudan", C.byref(desc), md, 1, 1, 0.0, ws.data_ptr(), ws.numel(),
                              q.data_ptr())
        for _ in range(args.warmup if mode != "fp32" else 1):
            f()
        ms = _time(f, args.steps if mode != "fp32" else 2, stream, torch)
        out[mode] = {"ms_per_solve": round(ms, 3), "quotes_per_s": round(NK / (ms * 1e-3), 1), "q": q.clone()}
        del ws
    # FP64 reference (outside the timed regions)
    d = lat.d
    cols = lat.cols.view(d, -1).long()
    vals = lat.vals.view(d, -1)
    mask = cols >= 0
    rows = torch.arange(d, device=dev).unsqueeze(1).expand_as(cols)
    Ld = torch.zeros(d, d, dtype=torch.float64, device=dev)
    Ld.index_put_((rows[mask], cols[mask]), vals[mask], accumulate=True)
    P = torch.eye(d, dtype=torch.float64, device=dev) + plan.dt * Ld
    del Ld
    for _ in range(plan.niter):
        P = P @ P
        P /= P.sum(dim=1, keepdim=True)
    ref = induction(P, torch.float64)
    del P
    for mode in out:
        out[mode]["max_abs_err_vs_fp64"] = float((out[mode].pop("q") - ref).abs().max().item())
    # plain FP32 arm: cuBLAS squaring with FP64 row renormalisation, FP32 induction products
    prev_tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False

    def fp32_arm():
        P = torch.zeros(d, d, dtype=torch.float32, device=dev)
        P.index_put_((rows[mask], cols[mask]), (plan.dt * vals[mask]).float(), accumulate=True)
        P.diagonal().add_(1.0)
        T = torch.empty_like(P)
        for _ in range(plan.niter):
            torch.mm(P, P, out=T)
            P, T = T, P
            P.mul_((1.0 / P.sum(dim=1, dtype=torch.float64)).float().unsqueeze(1))
        return induction(P, torch.float32)

    fp32_arm()
    torch.cuda.synchronize()
    ms32 = _time(fp32_arm, max(2, args.steps // 3), stream, torch)
    err32 = float((fp32_arm() - ref).abs().max().item())
    torch.backends.cuda.matmul.allow_tf32 = prev_tf32
    best = out["bf16x3"]
    return {"metric": "Bermudan put quotes/sec (backward induction on the SV d=6144 period kernel)",
            "value": best["quotes_per_s"], "unit": "quotes/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": best["ms_per_solve"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic",
            "config": {"workload": f"SV lattice d={d}, {NK} strikes, Bermudan puts exercisable every {PERIOD} y "
                                   f"to {PERIOD * NMAT} y", "niter": plan.niter, "products": NMAT},
            "max_abs_err_vs_fp64": best["max_abs_err_vs_fp64"], "modes": out,
            "fp32_cublas": {"quotes_per_s": round(NK / (ms32 * 1e-3), 1), "ms_per_solve": round(ms32, 3),
                            "max_abs_err_vs_fp64": err32},
            "speedup_vs_fp32_cublas": round(ms32 / best["ms_per_solve"], 2),
            "speedup_vs_fp32_simt": round(out["fp32"]["ms_per_solve"] / best["ms_per_solve"], 2),
            "speedup_vs_fp32": round(min(ms32, out["fp32"]["ms_per_solve"]) / best["ms_per_solve"], 2)}


def run_gemm(args):
    """The squaring GEMM alone (split-BF16, E-form: C = E.E + 2E in place) at size d, in the
    solve's form: B is E's own row-major parts, read as an MN-major operand.  --cta-pair 0
    runs the one-CTA 128 x 256 kernel instead of the 2-CTA pair kernel."""
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import bind_stream
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    lib = _lib.load()
    d = args.d
    lib.opb_set_cta_pair(args.cta_pair)
    Ah = torch.empty(d, d, dtype=torch.bfloat16, device=dev).normal_(0, 1e-3)
    Al = torch.empty_like(Ah).normal_(0, 1e-6)
    X = torch.empty(d, d, dtype=torch.float32, device=dev).normal_()
    rs = torch.empty(lib.opb_gemm_bf16x3_nparts(d, d) * d, dtype=torch.float64, device=dev)
    a = (d, d, d, Ah.data_ptr(), Al.data_ptr(), d, Ah.data_ptr(), Al.data_ptr(), d, 1.0, X.data_ptr(), 2.0,
         X.data_ptr(), d, rs.data_ptr())
    for _ in range(args.warmup):
        _lib.call("opb_gemm_bf16x3_kn", *a)
    ms = _time(lambda: _lib.call("opb_gemm_bf16x3_kn", *a), args.steps, torch.cuda.current_stream(dev), torch)
    _, peak, _, src = _peaks()
    tf = 3 * 2.0 * d ** 3 / (ms * 1e-3) / 1e12
    return {"metric": "split-BF16 GEMM MMA TFLOP/s", "value": round(tf, 1), "unit": "TFLOP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic",
            "config": {"workload": f"E-form squaring GEMM d={d}", "cta_pair": args.cta_pair},
            "frac_of_peak": round(tf / peak, 4),
            "peak_source": src}


def run_solve(args):
    """One SV lattice solve of a chosen grid (--sv-nx x --sv-nv states, config 1's parameters
    otherwise: 16 maturities x 128 strikes), CUDA-graph replay, in --mode; with
    --fused-max-d the row normalisation's form (fused into the epilogues up to that many
    states, a kernel after every product above)."""
    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import MODES, Lattice, bind_stream
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    stream = torch.cuda.current_stream(dev)
    sv = dict(SV, nx=args.sv_nx, nv=args.sv_nv)
    lat = Lattice.stoch_vol(**sv, device=dev)
    plan = lat.plan(PERIOD, DT0)
    strikes = torch.tensor(STRIKES, dtype=torch.float64, device=dev)
    mode = MODES[args.mode]
    ws = lat.workspace(NK, mode)
    q = torch.empty(NMAT, NK, dtype=torch.float64, device=dev)
    desc = lat.desc(plan, PERIOD, NMAT, strikes)

    def step():
        _lib.call("opb_lattice_solve", C.byref(desc), mode, ws.data_ptr(), ws.numel(), q.data_ptr(), None)
    for _ in range(args.warmup):
        step()
    g = _graph(step, dev, torch)
    g.replay()
    ms = _time(g.replay, args.steps, stream, torch)
    return {"metric": "priced quotes/sec, SV lattice solve (CUDA-graph replay)",
            "value": round(NMAT * NK / (ms * 1e-3), 1), "unit": "quotes/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.mode, "data": "synthetic",
            "config": {"workload": f"SV lattice {args.sv_nv} vol x {args.sv_nx} spot = {lat.d} states, "
                                   f"{plan.niter} squarings + {NMAT - 1} chains, {NK} strikes x {NMAT} maturities",
                       "fused_max_d": args.fused_max_d}}


def run_price(args):
    """The pricing / induction product alone at size d: V = P.G with P's two BF16 parts (d x d)
    against 128 payoff columns (two parts), three split products as K-slices whose FP32
    partials the caller sums (the form of the SV solve's 16 pricing products and of the
    Bermudan induction).  Algorithmic bytes: P's parts read once (4 d^2), the payoff parts
    (4 * 128 d) and the partials written (4 * 128 d per slice).  Beside it, a device copy
    moving the same number of bytes (read + write), timed the same way, as the bandwidth a
    transfer of this size reaches.  Inputs larger than L2 (151 MB)."""
    import ctypes

    import torch
    from oplib_b200 import _lib
    from oplib_b200.model import bind_stream
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    bind_stream(dev)
    lib = _lib.load()
    d, n = args.d, 128
    Ph = torch.empty(d, d, dtype=torch.bfloat16, device=dev).uniform_(0, 2.0 / d)
    Pl = (torch.empty(d, d, dtype=torch.float32, device=dev).uniform_(-1, 1) * 2.0 ** -9 / d).to(torch.bfloat16)
    Gh = torch.empty(n, d, dtype=torch.bfloat16, device=dev).uniform_(0, 1)
    Gl = (torch.empty(n, d, dtype=torch.float32, device=dev).uniform_(-1, 1) * 2.0 ** -9).to(torch.bfloat16)
    used = ctypes.c_int(0)
    C = torch.empty(4 * d * n, dtype=torch.float32, device=dev)
    call = lambda: _lib.call("opb_gemm_bf16x3_ksliced", d, n, d, Ph.data_ptr(), Pl.data_ptr(), d, Gh.data_ptr(),
                             Gl.data_ptr(), d, C.data_ptr(), n, 0, d * n, ctypes.byref(used))
    stream = torch.cuda.current_stream(dev)
    res = {}
    for _ in range(args.warmup):
        call()
    ms = _time(call, args.steps, stream, torch)
    nbytes = 4.0 * d * d + 4.0 * n * d + 4.0 * n * d * used.value
    src_b = torch.empty(int(nbytes) // 2, dtype=torch.uint8, device=dev)
    dst_b = torch.empty_like(src_b)
    for _ in range(args.warmup):
        dst_b.copy_(src_b)
    ms_copy = _time(lambda: dst_b.copy_(src_b), args.steps, stream, torch)
    hbm, _, _, src = _peaks()
    gbs = nbytes / (ms * 1e-3) / 1e9
    gbs_copy = 2 * src_b.numel() / (ms_copy * 1e-3) / 1e9
    return {"metric": "pricing product GB/s (P read once)", "value": round(gbs, 1), "unit": "GB/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3",
            "data": "synthetic (inputs larger than L2)",
            "config": {"workload": f"V = P.G, d={d}, 128 columns, {used.value} K-slices"},
            "frac_of_hbm": round(gbs / hbm, 4), "peak_source": src,
            "copy_same_bytes": {"GB/s": round(gbs_copy, 1), "us": round(ms_copy * 1e3, 2),
                                "frac_of_hbm": round(gbs_copy / hbm, 4)},
            "frac_of_copy_same_bytes": round(gbs / gbs_copy, 4),
            "us_per_launch": round(ms * 1e3, 2), "algorithmic_bytes": nbytes}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--mode", default="bf16x3", choices=["bf16x3", "fp16x3", "fp32", "fp32_plain"])
    ap.add_argument("--no-compare", dest="compare", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu", action="store_false")
    ap.add_argument("--nlat", type=int, default=None,
                    help="lattices for --workload batch (default 512), problems for --workload calibrate (default 64)")
    ap.add_argument("--train-lattices", type=int, default=2600, help="~2^21 training quotes after the vega filter")
    ap.add_argument("--members", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--workload", default="sv",
                    choices=["sv", "lv", "mc", "gemm", "gemv", "renorm", "batch", "surrogate", "calibrate",
                             "refbench", "bermudan", "price", "solve"],
                    help="sv = the headline SV lattice solve; the others are secondary measurements")
    ap.add_argument("--d", type=int, default=4096, help="matrix size for --workload gemm")
    ap.add_argument("--mc-steps", type=int, default=504,
                    help="--workload mc: steps per path (504 = two years of daily steps)")
    ap.add_argument("--sv-nx", type=int, default=128, help="--workload solve: spot states")
    ap.add_argument("--sv-nv", type=int, default=48, help="--workload solve: vol states")
    ap.add_argument("--fused-max-d", type=int, default=-1,
                    help="largest single lattice whose row normalisation is fused into the products' epilogues "
                         "(-1: the library's default)")
    ap.add_argument("--cta-pair", type=int, default=1, choices=[0, 1],
                    help="--workload gemm: 2-CTA pair kernel (1, the default) or one CTA per tile (0)")
    args = ap.parse_args()
    if args.nlat is None:
        args.nlat = 64 if args.workload == "calibrate" else 512
    if args.fused_max_d >= 0 and args.impl == "b200":
        from oplib_b200 import _lib
        _lib.call("opb_set_fused_normalisation", args.fused_max_d)
    if args.workload != "sv" and args.impl == "b200":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        launched = "LOCAL_RANK" in os.environ  # under torchrun (any world size)
        if launched:
            if args.workload not in ("mc", "batch"):
                raise SystemExit("only the sv, mc and batch workloads run under torchrun")
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        fn = {"lv": run_lv, "mc": run_mc, "gemm": run_gemm, "gemv": run_gemv, "renorm": run_renorm,
              "batch": run_batch_sharded if launched else run_batch, "surrogate": run_surrogate,
              "calibrate": run_calibrate, "refbench": run_refbench, "bermudan": run_bermudan,
              "price": run_price, "solve": run_solve}[args.workload]
        line = fn(args)
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps(line))
        if launched:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # The reference's own host FP64 path on the host cores (rank 0 only).  A step is one
        # product of the solve, a bounded sample of it (1/29 of a solve).  One whole solve runs
        # first, untimed (it also warms the BLAS threads); it keeps the inputs of the stages
        # the timed steps run, spread evenly over the solve, so that the sample weighs cheap
        # and dear products as a solve does.  value = quotes per solve x (timed products / 29)
        # / timed seconds.
        if rank != 0:
            return 0
        t0 = time.perf_counter()
        hs = HostSolve()
        pos = hs.positions(args.steps)
        t_full, _, inputs = hs.solve(keep=set(pos))
        for i in range(args.warmup):
            hs.run_stage(pos[i % len(pos)], inputs[pos[i % len(pos)]])
        ts = [hs.run_stage(p, inputs[p]) for p in pos]
        timed = sum(ts)
        v = round(NMAT * NK * (args.steps / hs.stages) / timed, 3)
        cb = {"value": v, "unit": "quotes/s", "cores": hs.nth, "kind": "port", "cpu_model": hs.model,
              "sample": f"{args.steps} timed products of the reference's host FP64 solve of the SV lattice at stage "
                        f"positions spread over the {hs.stages} of a solve (U0 = I + dt L, {hs.niter} squarings, "
                        f"{NMAT - 1} chain products; payoff products with their P_m), inputs from one untimed "
                        f"whole solve; torch-CPU/MKL DGEMM, {hs.nth} threads, denormals flushed: {hs.ftz}; "
                        f"value = {NMAT * NK} quotes x (timed products / {hs.stages}) / timed seconds"}
        line = {"impl": "reference", "metric": SV_METRIC, "value": v,
                "unit": "quotes/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(timed / args.steps * 1e3, 1), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": sv_config(args.mode, 1),
                "cpu_baseline": cb, "e2e": {"value": v, "unit": "quotes/s", "h2d_bytes_per_step": 0,
                                            "d2h_bytes_per_step": 0},
                "step_s_min_max": [round(min(ts), 3), round(max(ts), 3)],
                "untimed_whole_solve_s": round(t_full, 2),
                "wall_s": round(time.perf_counter() - t0, 1)}
        print(json.dumps(line))
        return 0

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    out = run_b200(args, rank, world, local_rank)
    if rank == 0:
        if args.compare and world == 1:
            try:
                out["config3_sweep"] = sweep_summary(args)
            except Exception as e:  # a secondary figure must not cost the headline line
                out["config3_sweep"] = {"error": f"{type(e).__name__}: {e}"[:300]}
            try:
                out["config2_mc"] = mc_summary(args)
            except Exception as e:
                out["config2_mc"] = {"error": f"{type(e).__name__}: {e}"[:300]}
            try:
                out["config4_surrogate"] = surrogate_summary(args)
            except Exception as e:
                out["config4_surrogate"] = {"error": f"{type(e).__name__}: {e}"[:300]}
        if args.cpu:
            out["cpu_baseline"] = cpu_baseline()
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
