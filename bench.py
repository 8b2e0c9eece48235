#!/usr/bin/env python
"""Benchmark of the Bloch-McConnell forward model on B200: Z-spectra per second.

Workload (the batched forward-simulation configuration): 65,536 voxels of water + four CEST pools
(amide 3.5, amine 2.0, hydroxyl 1.0, NOE -3.5 ppm) + a super-Lorentzian MT pool (-2.5 ppm) at 3 T;
per voxel k and f of every CEST pool, water T1, water T2 and the B0 shift drawn uniformly (seeded);
a pulse train of 20 Gaussian pulses (50 ms, 200 samples each, 1 uT peak) each followed by a 5 ms
gap, then a spoiler, a 3 s recovery and the readout (4,023 events), at 101 offsets from -10 to
10 ppm. One step = the whole forward pass over every voxel and offset. Synthetic, seeded data.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`value` is device-resident throughput (inputs already in HBM); `e2e` is the same metric through the
C ABI with host buffers, host<->device copies inside the timed region. Under torchrun every rank
simulates its own 65,536 voxels (weak scaling, no collective on the data path) and the step time is
the max over ranks. `--impl reference` times the CPU oracle (oracle/bmc_oracle.c, float64 Pade-13
scaling and squaring, OpenMP on every host core) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "bmc-jax_b200"))

GAMMA = 267.5153
B0 = 3.0
POOLS = [  # (dw ppm, T1 s, T2 s): amide, amine, hydroxyl (amide's relaxation), NOE, and a fifth pool
    (3.5, 1.0, 0.1), (2.0, 1.0, 0.1), (1.0, 1.0, 0.1), (-3.5, 1.3, 0.005), (1.9, 1.0, 0.03)]


def pulse_train(n_off=101, n_pulses=20, n_samples=200, tp=0.05, gap=0.005, recovery=3.0, b1_uT=1.0,
                recovery_first=False):
    """The event table (type, dt, rf_amp, rf_phase, rf_freq, adc_idx), each (n_off, n_events)."""
    t = (np.arange(n_samples) + 0.5) / n_samples
    shape = np.exp(-((t - 0.5) ** 2) / (2 * (1.0 / 6.0) ** 2))
    amp = b1_uT * GAMMA / (2 * np.pi) * shape / shape.max()
    T, DT, A = [], [], []
    if recovery_first:
        T.append(0); DT.append(recovery); A.append(0.0)
    for _ in range(n_pulses):
        T += [1] * n_samples; DT += [tp / n_samples] * n_samples; A += list(amp)
        T.append(0); DT.append(gap); A.append(0.0)
    T.append(4); DT.append(0.0); A.append(0.0)
    if not recovery_first:
        T.append(0); DT.append(recovery); A.append(0.0)
    T.append(3); DT.append(0.0); A.append(0.0)
    ne = len(T)
    freq = np.linspace(-10.0, 10.0, n_off) * 42.5764 * B0
    typ = np.tile(np.int32(T), (n_off, 1))
    rf = np.where(typ == 1, freq[:, None], 0.0)
    adc = np.where(typ == 3, 0, -1).astype(np.int32)
    return (typ, np.tile(np.float64(DT), (n_off, 1)), np.tile(np.float64(A), (n_off, 1)),
            np.zeros((n_off, ne)), rf.astype(np.float64), adc)


def voxel_params(n_vox, n_cest=4, seed=0):
    """(params [13 + 5 n_cest][n_vox] in the C ABI layout, M0 [n_vox][N]) for seeded random voxels."""
    rng = np.random.default_rng(seed)
    pools = POOLS[:n_cest]
    rows = [1.0 / rng.uniform(0.8, 2.5, n_vox), 1.0 / rng.uniform(0.03, 0.12, n_vox), np.ones(n_vox)]
    k = rng.uniform(10.0, 5000.0, (n_cest, n_vox))
    f = rng.uniform(1e-5, 0.02, (n_cest, n_vox))
    rows += list(k) + list(f)
    rows += [np.full(n_vox, p[0]) for p in pools]
    rows += [np.full(n_vox, 1.0 / p[1]) for p in pools]
    rows += [np.full(n_vox, 1.0 / p[2]) for p in pools]
    rows += [np.full(n_vox, 30.0), np.full(n_vox, 0.05), np.full(n_vox, -2.5), np.full(n_vox, 1.0),
             np.full(n_vox, 1.0 / 1e-5), np.full(n_vox, 2.0), np.full(n_vox, B0), np.full(n_vox, GAMMA),
             rng.uniform(-0.3, 0.3, n_vox), np.ones(n_vox)]
    P = np.ascontiguousarray(np.stack(rows), np.float64)
    N = 3 * (1 + n_cest) + 1
    M0 = np.zeros((n_vox, N))
    M0[:, 2 * (1 + n_cest)] = 1.0
    M0[:, 2 * (1 + n_cest) + 1:3 * (1 + n_cest)] = f.T
    M0[:, 3 * (1 + n_cest)] = 0.05
    return P, M0


# ------------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx = float(c[2])
            except ValueError:
                continue
            for nm, val in zip(names, c[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x: float, device=None) -> float:
    """The largest value of x over every rank (the step time of the slowest GPU); x itself alone."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seed(rank: int) -> int:
    """Every rank simulates its own voxels (weak scaling): distinct seeds per rank."""
    return 1000 + rank


# Used when MEASURED_PEAKS.json (written on the GPU machines) is absent: an earlier measurement on the same
# pool of B200s -- a STREAM-style copy and a burst cuBLAS bf16 GEMM.
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def measured_peaks():
    """The measured HBM and bf16 peaks (MEASURED_PEAKS.json), or FALLBACK_PEAKS marked as the fallback."""
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        d.setdefault("source", "MEASURED_PEAKS.json")
        return d
    except (OSError, ValueError):
        return dict(FALLBACK_PEAKS)


# ------------------------------------------------------------------------------------------------
# CPU baseline: the C oracle on the host cores, bounded sample
# ------------------------------------------------------------------------------------------------
def cpu_baseline(P, M0, ev, n_cest, budget_s=15.0, kind="port", return_z=False):
    sys.path.insert(0, str(ROOT / "oracle"))
    import bmc_oracle as O
    mz = 2 * (1 + n_cest)
    events = O.Events(*ev)
    threads = O.c_oracle().oracle_threads()
    n_off = ev[0].shape[0]
    # calibrate on a fraction of one voxel's offsets, then size the sample to the budget
    cal_off = max(threads, 8)
    t = time.perf_counter()
    sub = O.Events(*[a[:cal_off] for a in events])
    O.c_simulate_z(P[:, :1], sub, M0[:1], n_cest, mz, threads)
    per_chain = (time.perf_counter() - t) / cal_off
    n_vox = max(1, int(budget_s / max(per_chain * n_off, 1e-9)))
    n_vox = min(n_vox, P.shape[1])
    t = time.perf_counter()
    z = O.c_simulate_z(P[:, :n_vox], events, M0[:n_vox], n_cest, mz, threads)
    el = time.perf_counter() - t
    line = {"value": n_vox / el, "unit": "Z-spectra/s", "cores": threads, "kind": kind,
            "sample": f"{n_vox} voxels x {n_off} offsets x {ev[0].shape[1]} events, float64 Pade-13 "
                      f"expm per event (oracle/bmc_oracle.c, OpenMP), {el:.1f} s"}
    return (line, z) if return_z else line


def oracle_check(P, M0, ev, n_cest, z_gpu, n_vox=8):
    """max |dZ| of the first n_vox voxels of a timed output against the float64 C oracle (after timing)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import bmc_oracle as O
    want = O.c_simulate_z(P[:, :n_vox], O.Events(*ev), M0[:n_vox], n_cest, 2 * (1 + n_cest))
    return float(np.max(np.abs(np.asarray(z_gpu)[:n_vox] - want)))


# ------------------------------------------------------------------------------------------------
# DRAM bytes per chain of chain_kernel from one ncu capture of a 2,048-voxel x 101-offset launch of the
# default workload (float64: 22.0 MB read + 37.6 MB written; mixed: 22.4 MB + 23.9 MB; almost all of it
# register-spill traffic); it grows with the number of chains a launch runs. Keyed by (CEST pools,
# precision, pulses).
NCU_BYTES_PER_CHAIN = {(4, 0, 20): (21.957632e6 + 37.630464e6) / (2048 * 101),
                       (4, 2, 20): (22.438656e6 + 23.910656e6) / (2048 * 101)}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from bmc_b200 import _lib
    from bmc_b200.simulation import DeviceEvents, problem
    import ctypes as C

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    nc = args.pools
    N = 3 * (1 + nc) + 1
    mz = 2 * (1 + nc)
    P, M0 = voxel_params(args.voxels, nc, seed=rank_seed(rank))
    ev = pulse_train(args.offsets, n_pulses=args.pulses)
    n_off, n_ev = ev[0].shape
    nv = args.voxels
    prec = {"f64": _lib.F64, "f32": _lib.F32, "mixed": _lib.MIXED}[args.precision]

    # host (pinned) and device copies
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hP, hM = pin(P), pin(M0)
    hev = [pin(a) for a in ev]
    dP, dM = hP.to(dev), hM.to(dev)
    dev_ev = DeviceEvents.from_tensors(*[x.to(dev) for x in hev])
    dZ = torch.empty((nv, n_off), dtype=torch.float64, device=dev)
    hZ = torch.empty((nv, n_off), dtype=torch.float64).pin_memory()
    pr = problem(nv, n_off, n_ev, nc, mz, prec)
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev)
    sh = C.c_void_p(stream.cuda_stream)

    sp, keep_sp, spread_cfg = None, None, None
    if args.spread_nodes:
        # configuration 5: every voxel a Gauss-Hermite B0 spread of sigma = 0.1 ppm at 3 T (12.77 Hz)
        from bmc_b200.simulation import B0Spread
        sigma_hz = 0.1 * 42.5764 * B0
        u, w = B0Spread(sigma_hz, "gauss", args.spread_nodes).nodes_weights()
        sig = torch.full((nv,), sigma_hz, dtype=torch.float64, device=dev)
        sp, keep_sp = _lib.spread_struct(u, w, sig)
        spread_cfg = {"shape": "gauss", "nodes": args.spread_nodes, "sigma_hz": sigma_hz}

    def step(params=dP, m0=dM, evs=dev_ev, out=dZ):
        _lib.check(L.bmc_simulate(pr, C.c_void_p(params.data_ptr()), evs.struct, C.c_void_p(m0.data_ptr()), sp,
                                  C.c_void_p(out.data_ptr()), sh))

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # 256 MB > L2 (126 MB)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    # executed work of one launch (deterministic), from the kernel's own counters
    work = torch.zeros(5, dtype=torch.int64, device=dev)
    _lib.check(L.bmc_simulate_counted(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct, C.c_void_p(dM.data_ptr()),
                                      sp, C.c_void_p(dZ.data_ptr()), C.c_void_p(work.data_ptr()), sh))
    torch.cuda.synchronize(dev)
    terms, hcols, squar, executed, terms32 = [int(x) for x in work.cpu()]
    nnz = 12 + 15 * nc                                   # nonzeros of A (+ C folded into term 1)
    flop_term = 2 * nnz + 2 * N                          # operator product + scaling + accumulation
    NA = N + 1
    # FLOPs by pipe: the Taylor terms formed in float32 on the FP32 pipe, the rest (and the dense path)
    # on the FP64 pipe
    flops32 = terms32 * flop_term
    flops64 = (terms - terms32) * flop_term + hcols * flop_term + squar * 2.0 * N * N * NA
    flops = flops32 + flops64

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler = ClockSampler(local_rank)
    sampler.start()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)                                 # L2 flush between timed iterations (not timed)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    ms = max_over_ranks(float(np.mean(times)), dev)
    if world > 1:
        dist.barrier()

    # end to end: host buffers in, Z back to the host, copies inside the timed region (at most 5 steps: the
    # copies add ~15 ms to a ~4 s step, so more steps would only lengthen the run)
    e2e = []
    e2e_steps = max(1, min(args.steps, 5))
    for _ in range(e2e_steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dP.copy_(hP, non_blocking=True)
        dM.copy_(hM, non_blocking=True)
        for d, h in zip(dev_ev.t, hev):
            d.copy_(h, non_blocking=True)
        step()
        hZ.copy_(dZ, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        e2e.append(e0.elapsed_time(e1))
    e2e_ms = max_over_ranks(float(np.mean(e2e)), dev)
    h2d = sum(x.numel() * x.element_size() for x in [hP, hM] + hev)
    d2h = hZ.numel() * hZ.element_size()

    # FMA peaks of this GPU, measured now (burst, like a kernel timed alone), FP64 and FP32 pipes; the
    # roofline of a launch whose work runs on both is the time the two shares take at their peaks
    best = fp64_peak()
    best32 = fma_peak(_lib.F32)
    t_ideal = flops64 / (best * 1e12) + flops32 / (best32 * 1e12)
    peak_eff = flops / t_ideal / 1e12 if t_ideal > 0 else best
    achieved = flops / (ms * 1e-3) / 1e12
    value = world * nv / (ms * 1e-3)
    f32_err = None
    if prec != _lib.F64:
        # accuracy of the float32 kernel: the same voxels through the float64 kernel (after timing)
        ns = min(nv, 4096)
        z64 = torch.empty((ns, n_off), dtype=torch.float64, device=dev)
        pr64 = problem(ns, n_off, n_ev, nc, mz, _lib.F64)
        dP_s, dM_s = dP[:, :ns].contiguous(), dM[:ns].contiguous()
        _lib.check(L.bmc_simulate(pr64, C.c_void_p(dP_s.data_ptr()), dev_ev.struct, C.c_void_p(dM_s.data_ptr()), sp,
                                  C.c_void_p(z64.data_ptr()), sh))
        step()
        torch.cuda.synchronize(dev)
        f32_err = {"voxels": ns, "max_abs_err_vs_f64": float((dZ[:ns] - z64).abs().max().item())}
    traffic, traffic_src = None, "no ncu capture of this configuration"
    if (nc, prec, args.pulses) in NCU_BYTES_PER_CHAIN and not args.spread_nodes:
        traffic = NCU_BYTES_PER_CHAIN[(nc, prec, args.pulses)] * nv * n_off
        traffic_src = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one 2,048-voxel launch, scaled by "
                       "the chains of this launch")
    line = {
        "metric": "Z-spectra/s (batched forward simulation)", "value": value, "unit": "Z-spectra/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {_lib.F64: "f64", _lib.F32: "f32", _lib.MIXED: "f64 state + f32 Taylor tail (mixed)"}[prec],
        "data": "synthetic (seeded)",
        "config": {"workload": f"forward simulation: {nv} voxels per GPU x {n_off} offsets x {n_ev} events, "
                               f"water + {nc} CEST pools + super-Lorentzian MT (state {N}, augmented {NA}), "
                               f"20 Gaussian 50 ms pulses + 5 ms gaps, spoiler, 3 s recovery, ADC",
                   "voxels_per_gpu": nv, "offsets": n_off, "events": n_ev, "pools": nc,
                   "parallelism": f"dp{world} (voxels sharded, no collective)",
                   "l2": "flushed between timed steps (256 MB write, untimed)", "b0_spread": spread_cfg,
                   "float32_accuracy": f32_err,
                   "taylor_tail": {_lib.F64: "Taylor terms below 1e-6 of the state (bound theta^k/k!) formed in "
                                             "float32, summed into the float64 state once per sub-step; "
                                             "truncation 1e-13 per sub-step",
                                   _lib.MIXED: "the first Taylor term of every sub-step in float64 (more where their "
                                               "bound theta^k/k! exceeds 3x the state), later terms in float32, "
                                               "summed into the float64 state once per sub-step; truncation 1e-9 "
                                               "per sub-step",
                                   _lib.F32: "all Taylor terms and the state in float32; truncation 2^-24"}[prec]},
        "e2e": {"value": world * nv / (e2e_ms * 1e-3), "unit": "Z-spectra/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms, "steps": e2e_steps},
        "roofline": {"bound": "fp64+fp32 fma", "achieved": achieved, "peak": peak_eff, "unit": "TFLOP/s",
                     "frac": achieved / peak_eff if peak_eff else None,
                     "traffic": traffic, "traffic_unit": "bytes per launch",
                     "traffic_source": traffic_src, "kernel": "chain_kernel",
                     "flops_per_launch": flops, "flops_fp64_pipe": flops64, "flops_fp32_pipe": flops32,
                     "peak_fp64": best, "peak_fp32": best32,
                     "frac_fp64_equivalent": achieved / best if best else None,
                     "taylor_terms": terms, "taylor_terms_float32": terms32, "taylor_terms_executed": executed,
                     "dense_columns": hcols, "dense_squarings": squar,
                     # the reference's work for the same result: one dense Pade-13 exponential of the
                     # augmented matrix per event and chain (6 products and an LU solve with NA right-hand
                     # sides, (6 + 4/3) 2 NA^3 FLOPs; its squarings left out, so a lower bound)
                     "reference_equivalent": {
                         "what": f"dense Pade-13 expm of the {NA}x{NA} augmented matrix per event (no squarings: "
                                 "a lower bound), as simulation/expm.py computes it",
                         "flops_per_event": (6 + 4 / 3) * 2 * NA ** 3,
                         "events_per_launch": nv * n_off * n_ev,
                         "tflops": (6 + 4 / 3) * 2 * NA ** 3 * nv * n_off * n_ev / (ms * 1e-3) / 1e12},
                     "peak_source": ("measured in this run: FMA-chain probe kernel (bmc_probe_fma_peak), burst; "
                                     "peak = the two pipes' peaks weighted by this launch's FLOPs on each "
                                     "(time of the FP64 share at the FP64 peak plus the FP32 share at the "
                                     "FP32 peak)")},
        "clocks": clocks,
        "gpu_launches": 2 * args.steps,
    }
    # the float64 kernel on the same inputs, timed the same way over at most three steps, for comparison
    if prec != _lib.F64 and not args.spread_nodes:
        pr64 = problem(nv, n_off, n_ev, nc, mz, _lib.F64)
        z64 = torch.empty_like(dZ)
        call64 = lambda: _lib.check(L.bmc_simulate(pr64, C.c_void_p(dP.data_ptr()), dev_ev.struct,
                                                   C.c_void_p(dM.data_ptr()), sp, C.c_void_p(z64.data_ptr()), sh))
        call64()
        t64 = []
        for _ in range(max(1, min(args.steps, 3))):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call64()
            e1.record(stream)
            e1.synchronize()
            t64.append(e0.elapsed_time(e1))
        ms64 = max_over_ranks(float(np.mean(t64)), dev)
        line["f64_kernel"] = {"value": world * nv / (ms64 * 1e-3), "unit": "Z-spectra/s", "ms_per_step": ms64,
                              "steps": len(t64), "max_abs_diff_vs_this_line": float((dZ - z64).abs().max().item())}
        del z64
    # the timed output itself against the float64 C oracle, on its first voxels (after timing); with the
    # CPU baseline, on the voxels the baseline simulated
    z_host = hZ.numpy()
    if rank == 0 and world == 1 and not args.no_cpu and not args.spread_nodes:
        line["cpu_baseline"], z_cpu = cpu_baseline(P, M0, ev, nc, budget_s=args.cpu_budget, return_z=True)
        n_chk = z_cpu.shape[0]
        err = float(np.max(np.abs(z_host[:n_chk] - z_cpu)))
    elif not args.spread_nodes:
        n_chk = min(nv, 4)
        err = oracle_check(P, M0, ev, nc, z_host, n_chk)
    else:
        n_chk, err = 0, None
    line["config"]["oracle_check"] = {"voxels": n_chk, "offsets": n_off,
                                      "max_abs_err_vs_float64_oracle": err,
                                      "oracle": "oracle/bmc_oracle.c (float64 Pade-13 expm per event)"}
    if world == 1 and not args.no_fit and not args.spread_nodes:
        line["fit"] = warm_vs_plain(args, rank, local_rank, peak_fp64=best)
    return line


def quesp_ladder(n_ppm=61, b1s=(0.5, 1.0, 2.0, 4.0), tsat=2.0, b0=3.0):
    """The configuration-1 sequence: one CW block per offset then the ADC, four rungs stacked."""
    ppm = np.linspace(-6.0, 6.0, n_ppm)
    rows = []
    for b1 in b1s:
        amp = b1 * GAMMA / (2 * np.pi)
        fr = ppm * 42.5764 * b0
        rows.append((np.tile(np.int32([1, 3]), (n_ppm, 1)), np.tile([tsat, 0.0], (n_ppm, 1)),
                     np.tile([amp, 0.0], (n_ppm, 1)), np.zeros((n_ppm, 2)),
                     np.stack([fr, np.zeros(n_ppm)], axis=1), np.tile(np.int32([-1, 0]), (n_ppm, 1))))
    return tuple(np.ascontiguousarray(np.concatenate([r[i] for r in rows])) for i in range(6))


def run_fit(args, rank, world, local_rank):
    """Fitted voxels/s: (k, f) of an amide pool (configuration 1's model at 3 T) from (300, 5e-4),
    30 LM iterations on the device, noise-free data; a voxel counts as fitted when both parameters are
    within 1% of the truth that made its data."""
    import torch
    import ctypes as C
    from bmc_b200 import _lib
    from bmc_b200.simulation import DeviceEvents, problem
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    n = args.voxels
    rng = np.random.default_rng(rank_seed(rank))
    k_true = rng.uniform(20.0, 1000.0, n)
    f_true = rng.uniform(3e-4, 3e-3, n)
    rows = [np.full(n, 1 / 1.3), np.full(n, 1 / 0.05), np.ones(n), k_true, f_true, np.full(n, 3.5),
            np.full(n, 1 / 1.3), np.full(n, 1 / 0.1), np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n),
            np.ones(n), np.zeros(n), np.full(n, B0), np.full(n, GAMMA), np.zeros(n), np.ones(n)]
    P = np.ascontiguousarray(np.stack(rows))
    M0 = np.zeros((n, 7)); M0[:, 4] = 1.0; M0[:, 5] = f_true
    ev = quesp_ladder()
    n_off, n_ev = ev[0].shape
    dev_ev = DeviceEvents.from_tensors(*[torch.as_tensor(a).to(dev) for a in ev])
    dP, dM = torch.as_tensor(P).to(dev), torch.as_tensor(M0).to(dev)
    L = _lib.lib()
    sh = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    pr = problem(n, n_off, n_ev, 1, 4, _lib.F64)
    z = torch.empty((n, n_off), dtype=torch.float64, device=dev)
    _lib.check(L.bmc_simulate(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct, C.c_void_p(dM.data_ptr()), None,
                              C.c_void_p(z.data_ptr()), sh))
    spec = _lib.FitSpecC()
    spec.n_params, spec.n_iter, spec.lam0 = 2, 30, 1e-2
    for p, (row, sc, lo, hi) in enumerate([(3, 100.0, 5.0, 5000.0), (4, 1e-3, 1e-6, 0.05)]):
        spec.field_row[p], spec.mode[p], spec.scale[p] = row, 0, sc
        spec.lo[p], spec.hi[p] = lo / sc, hi / sc
    x0 = torch.tensor(np.tile([3.0, 0.5], (n, 1)), dtype=torch.float64, device=dev)
    xo = torch.empty((n, 2), dtype=torch.float64, device=dev)

    def step():
        _lib.check(L.bmc_lm_fit(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct, C.c_void_p(dM.data_ptr()), None, spec,
                                C.c_void_p(z.data_ptr()), C.c_void_p(x0.data_ptr()), C.c_void_p(xo.data_ptr()),
                                None, None, sh))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    times = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = max_over_ranks(float(np.mean(times)), dev)
    x = xo.cpu().numpy() * np.array([100.0, 1e-3])
    ok = (np.abs(x[:, 0] / k_true - 1) <= 0.01) & (np.abs(x[:, 1] / f_true - 1) <= 0.01)
    return {"metric": "fitted voxels/s at <=1% param err (plain LM, device)", "value": world * n * ok.mean() / (ms * 1e-3),
            "unit": "voxels/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded), noise-free",
            "config": {"workload": f"LM fit of (k, f), amide pool at 3 T, QUESP ladder 4 x 61 CW offsets (2 s), "
                                   f"{n} voxels per GPU, 30 iterations from (300, 5e-4)",
                       "fraction_within_1pct": float(ok.mean()), "voxels_per_gpu": n}}


PHANTOM = ROOT / "tests" / "golden" / "phantom"
PUBLISHED_S = {"phantom08": 15 * 60.0, "phantom09": 15 * 60.0, "phantom10": 2 * 3600.0,   # 1x RTX 3070
               "phantom11": 3.5 * 3600.0}


def phantom_data(tubes=None):
    """The shipped phantom measurement (tests/golden/phantom), optionally only the tubes with a pool."""
    with np.load(PHANTOM / "phantom_7tubes.npz", allow_pickle=True) as d:
        data = {k: d[k] for k in d.files}
    if tubes == "pool":
        idx = np.flatnonzero(np.isfinite(data["vial_dw"]))
        per = ("Z_quesp", "Z_quest", "vial_names", "vial_dw", "R1", "b0_hz", "rel_b1", "noise_quesp", "noise_quest")
        data = {k: (v[idx] if k in per else v) for k, v in data.items()}
    return data


def phantom_params(d, pool_t2_s=0.010):
    """Every tube as one batched SimParams: measured water R1, B0 and B1 per tube, PBS water R2 for all,
    the CEST pool at its shift with T2 pool_t2_s (k and f are placeholders the fit replaces)."""
    from bmc_b200.simulation import SimParams
    n = len(d["vial_names"])
    one = np.ones(n)
    pool = np.isfinite(d["vial_dw"])
    b0 = float(d["b0_T"])
    return SimParams(water_r1=d["R1"].astype(float), water_r2=float(d["water_r2"]) * one, water_f=one,
                     cest_k=np.where(pool, 900.0, 0.0)[:, None], cest_f=np.where(pool, 0.008, 0.0)[:, None],
                     cest_dw=np.where(pool, d["vial_dw"], 0.0)[:, None].astype(float), cest_r1=one[:, None],
                     cest_r2=(one / pool_t2_s)[:, None], mt_k=0 * one, mt_f=0 * one, mt_dw=0 * one,
                     mt_r1=0 * one, mt_r2=one, mt_lineshape=np.zeros(n, np.int32), b0=b0 * one,
                     gamma=267.5153 * one, b0_inhom=d["b0_hz"] / (42.5764 * b0), rel_b1=d["rel_b1"].astype(float))


def phantom_events(stem, keep):
    """One rung's converted sequence, the -300 ppm reference row dropped, offsets masked by keep."""
    from bmc_b200.simulation import SimEvent
    with np.load(PHANTOM / f"{stem}_events.npz") as d:
        ev = SimEvent(*[np.asarray(d[f])[1:] for f in SimEvent._fields])
    return SimEvent(*[a[keep] for a in ev])


def run_phantom(args):
    """Tutorials 08 (QUESP fit), 09 (QUEST fit), 10 (joint fit: shared water R2 factor, M_start and a
    15-node B0 spread) and 11 (the joint fit again with one B1 factor per rung) of the reference on the
    shipped phantom data, through bmc_b200's public API; the wall time of the fit calls, host<->device
    traffic included, against the published RTX 3070 runtime."""
    import torch
    from dataclasses import replace
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam, fit, fit_joint
    from bmc_b200.simulation import initial_state, SimParams, B0Spread
    torch.cuda.init()
    w = args.workload

    def ladder_for(d, rungs, kind):
        p = phantom_params(d)
        n = len(d["vial_names"])
        m0 = np.stack([initial_state(SimParams(*[np.asarray(v)[i] for v in p]), float(d["m_start"])) for i in range(n)])
        keep = np.abs(d["ppm"]) >= 1.0
        stems = ([f"quesp_sim_b1_{('%g' % b).replace('.', 'p')}uT" for b in rungs] if kind == "quesp" else
                 [f"quest_sim_tsat_{('%g' % t).replace('.', 'p')}s" for t in rungs])
        lad = Experiment.stack([Experiment(p, phantom_events(s, keep), m0, 4) for s in stems])
        Z = d["Z_" + kind][:, :, keep].reshape(n, -1)
        return lad, Z, int(keep.sum())

    K = FreeParam("k", "cest_k", 0, scale=1000.0, lo=5.0, hi=2000.0, x0=300.0)
    F = FreeParam("f", "cest_f", 0, scale=0.01, lo=1e-5, hi=0.03, x0=0.008)
    T2 = FreeParam("r2p", "cest_r2", 0, scale=100.0, lo=10.0, hi=1000.0, x0=100.0)
    d6 = phantom_data("pool")
    kind = "quest" if w == "phantom09" else "quesp"
    rungs = d6["tsat_s"] if kind == "quest" else d6["b1_levels_uT"]
    lad6, Z6, n_per = ladder_for(d6, rungs, kind)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain = fit(lad6, FitSpec([K, F, T2]), Z6, n_iter=60, n_per_block=n_per)
    t_plain = time.perf_counter() - t0
    out = {"fit_s": t_plain, "tubes": [str(s) for s in d6["vial_names"]], "k": plain["k"].tolist(),
           "f": plain["f"].tolist(), "t2_pool_ms": (1e3 / plain["r2p"]).tolist(),
           "rms_over_noise": (plain.rms / d6["noise_" + kind]).tolist(),
           "points": int(Z6.shape[1]), "events": lad6.n_events}
    value = t_plain
    if w in ("phantom10", "phantom11"):
        d7 = phantom_data()
        pool = tuple(int(i) for i in np.flatnonzero(np.isfinite(d7["vial_dw"])))
        Kp, Fp, T2p = (replace(s, samples=pool) for s in (K, F, T2))
        R2F = FreeParam("r2w", "water_r2", None, scale=1.0, lo=0.5, hi=2.0, x0=1.0, scope="shared", mode="factor")
        MS = FreeParam("m_start", "m_start", None, scale=1.0, lo=0.2, hi=1.0, x0=float(d7["m_start"]), scope="shared")
        SIG = FreeParam("sigma", "b0_spread", None, scale=10.0, lo=0.0, hi=8.0, x0=5.0, scope="shared")
        spec = FitSpec([Kp, Fp, T2p, R2F, MS, SIG])
        x0 = np.tile([s.x0 for s in spec.slots], (7, 1))
        x0[list(pool), :3] = plain.x
        lad7, Z7, _ = ladder_for(d7, d7["b1_levels_uT"], "quesp")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        joint = fit_joint(lad7, spec, Z7, n_iter=12, n_per_block=n_per, x0_phys=x0, spread=B0Spread(nodes=15))
        t_joint = time.perf_counter() - t0
        value = t_plain + t_joint
        out.update(joint_s=t_joint, r2w=float(joint["r2w"][0]), m_start=float(joint["m_start"][0]),
                   sigma_hz=float(joint["sigma"][0]), joint_cost=[float(joint.cost[0]), float(joint.cost[-1])])
        if w == "phantom11":
            # tutorial 11: the same joint fit with one B1 factor per rung, shared by the tubes, from step 2
            B1R = FreeParam("b1", "rel_b1", None, scale=1.0, lo=0.7, hi=1.3, x0=1.0, scope="block", mode="factor")
            x1 = np.column_stack([joint.x, np.ones(joint.x.shape[0])])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            rung = fit_joint(lad7, FitSpec([Kp, Fp, T2p, R2F, MS, SIG, B1R]), Z7, n_iter=12, n_per_block=n_per,
                             x0_phys=x1, spread=B0Spread(nodes=15), block_jacobian="split")
            t_rung = time.perf_counter() - t0
            value += t_rung
            out.update(rung_s=t_rung, b1_per_rung=np.asarray(rung.blocks["b1"]["x"]).reshape(-1).tolist(),
                       rung_cost=[float(rung.cost[0]), float(rung.cost[-1])])
    pub = PUBLISHED_S[w]
    return {"metric": f"wall time of the reference's tutorial {w[-2:]} fit (public API, end to end)", "value": value,
            "unit": "s", "n_gpus": 1, "higher_is_better": False, "vs_baseline": value / pub,
            "published_s": pub, "published_on": "1x RTX 3070 (examples/README.md)", "dtype": "f64",
            "data": "the reference's shipped phantom measurement", "config": {"workload": w, **out}}


def run_reference(args):
    nc = args.pools
    P, M0 = voxel_params(max(args.voxels, 1), nc, seed=1000)
    ev = pulse_train(args.offsets, n_pulses=args.pulses)
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(P, M0, ev, nc, budget_s=2.0, kind="port")
    last = None
    for _ in range(args.steps):
        last = cpu_baseline(P, M0, ev, nc, budget_s=args.cpu_budget / max(args.steps, 1) * 2, kind="port")
        vals.append(last["value"])
    v = float(np.mean(vals))
    return {"impl": "reference", "metric": "Z-spectra/s (batched forward simulation)", "value": v,
            "unit": "Z-spectra/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": "same as the GPU arm, bounded sample per step", "pools": nc,
                       "offsets": args.offsets},
            "cpu_baseline": {**last, "value": v},
            "e2e": {"value": v, "unit": "Z-spectra/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ------------------------------------------------------------------------------------------------
# learned warm start (the MLP configuration): NN-warm vs plain LM on the configuration-1 ladder
# ------------------------------------------------------------------------------------------------
WARM_RANGES = {"k": (10.0, 5000.0), "f": (1e-5, 0.02), "r2w": (1 / 0.12, 1 / 0.03), "b0": (-0.3, 0.3)}


def warm_model(nc):
    """(Experiment, FitSpec, training ranges): water + nc CEST pools (+ the super-Lorentzian MT pool
    when nc >= 3) at 3 T, the configuration-1 ladder (4 x 61 CW offsets, 2 s), free (k, f) of amide
    and amine, water R2 and the B0 shift; water T1 1.3 s; the other pools fixed at mid-range values."""
    from bmc_b200.fitting import Experiment, FitSpec, FreeParam
    from bmc_b200.simulation import SimEvent, SimParams, initial_state
    pools = POOLS[:nc]
    k = np.array([300.0, 300.0, 1500.0, 20.0, 500.0][:nc])
    f = np.array([5e-4, 5e-4, 5e-3, 1e-2, 1e-3][:nc])
    mt = nc >= 3
    p = SimParams(water_r1=np.float64(1 / 1.3), water_r2=np.float64(1 / 0.07), water_f=np.float64(1.0),
                  cest_k=k, cest_f=f, cest_dw=np.array([q[0] for q in pools]),
                  cest_r1=np.array([1 / q[1] for q in pools]), cest_r2=np.array([1 / q[2] for q in pools]),
                  mt_k=np.float64(30.0 if mt else 0.0), mt_f=np.float64(0.05 if mt else 0.0),
                  mt_dw=np.float64(-2.5), mt_r1=np.float64(1.0), mt_r2=np.float64(1e5 if mt else 1.0),
                  mt_lineshape=np.int64(2 if mt else 0), b0=np.float64(B0), gamma=np.float64(GAMMA),
                  b0_inhom=np.float64(0.0), rel_b1=np.float64(1.0))
    ev = SimEvent(*quesp_ladder())
    exp = Experiment(p, ev, initial_state(p), 2 * (1 + nc))
    R = WARM_RANGES
    slots = [FreeParam("k_amide", "cest_k", 0, 100.0, 5.0, 6000.0, 300.0),
             FreeParam("f_amide", "cest_f", 0, 1e-3, 1e-6, 0.05, 5e-4)]
    ranges = [R["k"], R["f"]]
    if nc >= 2:
        slots += [FreeParam("k_amine", "cest_k", 1, 100.0, 5.0, 6000.0, 300.0),
                  FreeParam("f_amine", "cest_f", 1, 1e-3, 1e-6, 0.05, 5e-4)]
        ranges += [R["k"], R["f"]]
    slots += [FreeParam("r2w", "water_r2", None, 10.0, 5.0, 50.0, 1 / 0.07),
              FreeParam("b0", "b0_inhom", None, 0.1, -0.5, 0.5, 0.0)]
    ranges += [R["r2w"], R["b0"]]
    return exp, FitSpec(slots), ranges


def within_1pct(x, truth, names):
    """Every free parameter within 1% of the truth (the B0 shift, which crosses zero, within 0.003 ppm:
    1% of its 0.3 ppm half-range)."""
    ok = np.ones(x.shape[0], bool)
    for j, n in enumerate(names):
        if n == "b0":
            ok &= np.abs(x[:, j] - truth[:, j]) <= 0.003
        else:
            ok &= np.abs(x[:, j] / truth[:, j] - 1.0) <= 0.01
    return ok


def mlp_roofline(n_in, n_out, n_hidden=256, n_layers=3, batch=4096, steps=50, infer_batch=65536):
    """Tensor-core rate of the warm-start network's kernels, timed with CUDA events on a fresh network
    of the trained one's shape: training steps (forward with saved activations, backward, Adam) at
    `batch`, and one inference pass at `infer_batch`. Algorithmic FLOPs per sample: forward
    F = 2 (n_in H + (L-1) H^2 + H n_out); a training step 3F - 2 n_in H (every weight gradient, and
    every input gradient but the first layer's)."""
    import torch
    from bmc_b200.warmstart import MLP
    net = MLP(n_in, n_out, n_hidden, n_layers, seed=5)
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    x = torch.rand((batch, n_in), generator=g, device="cuda")
    t = torch.rand((batch, n_out), generator=g, device="cuda")
    xi = torch.rand((infer_batch, n_in), generator=g, device="cuda")

    d_step = torch.zeros(1, dtype=torch.int32, device="cuda")

    def step():
        net.forward(x, keep=True)
        net.backward(t)
        net.adam_dev(d_step, 1e-4)

    for _ in range(5):
        step()
    net.forward(xi)
    graph = torch.cuda.CUDAGraph()                 # what MLP.train replays
    with torch.cuda.graph(graph):
        step()
    graph.replay()
    torch.cuda.synchronize()
    e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    for _ in range(steps):
        graph.replay()
    e2.record()
    net.forward(xi)
    e3.record()
    e3.synchronize()
    del graph
    F = 2.0 * (n_in * n_hidden + (n_layers - 1) * n_hidden ** 2 + n_hidden * n_out)
    step_flops = (3 * F - 2.0 * n_in * n_hidden) * batch
    train_ms = e1.elapsed_time(e2) / steps
    train_tf = step_flops / (train_ms * 1e-3) / 1e12
    infer_tf = F * infer_batch / (e2.elapsed_time(e3) * 1e-3) / 1e12
    peaks = measured_peaks()
    peak = peaks.get("bf16_tflops")
    return {"bound": "tensor", "achieved": train_tf, "peak": peak, "unit": "TFLOP/s",
            "frac": train_tf / peak if peak else None, "traffic": None,
            "kernel": "gemm_kernel (tcgen05.mma kind::f16, bf16 in, fp32 TMEM accumulate)",
            "peak_source": f"bf16_tflops of {peaks['source']} (burst cuBLAS GEMM)",
            "train_step_ms": train_ms, "train_step": "one CUDA-graph replay (what MLP.train runs)",
            "train_step_ms_eager": e0.elapsed_time(e1) / steps, "train_batch": batch,
            "inference_tflops": infer_tf, "inference_ms": e2.elapsed_time(e3), "inference_batch": infer_batch,
            # input kernel + (L + 1) GEMMs forward; loss kernel + 2 (L + 1) GEMMs backward; Adam + step count
            "gpu_launches_per_train_step": 3 * n_layers + 6}


def dictionary_model():
    """(base SimParams, 30-row saturation schedule, M0, mz, grid) of the dictionary configuration: water
    + amide (3.5 ppm) + super-Lorentzian MT at 3 T; 30 rows, each a 1 s recovery, a 1 s CW block at the
    amide offset with B1 0.5..6 uT (a seeded schedule) and the readout; the grid sweeps amide k
    (64 log-spaced, 10..5000 1/s), amide f (32 log-spaced, 1e-5..0.02), water T1 (16, 0.8..2.5 s) and
    rel_b1 (32, 0.7..1.3): 1,048,576 entries."""
    from bmc_b200.simulation import SimEvent, SimParams, initial_state
    p = SimParams(water_r1=np.float64(1 / 1.3), water_r2=np.float64(1 / 0.07), water_f=np.float64(1.0),
                  cest_k=np.array([300.0]), cest_f=np.array([1e-3]), cest_dw=np.array([3.5]),
                  cest_r1=np.array([1.0]), cest_r2=np.array([10.0]), mt_k=np.float64(30.0),
                  mt_f=np.float64(0.05), mt_dw=np.float64(-2.5), mt_r1=np.float64(1.0), mt_r2=np.float64(1e5),
                  mt_lineshape=np.int64(2), b0=np.float64(B0), gamma=np.float64(GAMMA),
                  b0_inhom=np.float64(0.0), rel_b1=np.float64(1.0))
    rng = np.random.default_rng(30)
    b1 = rng.uniform(0.5, 6.0, 30)
    n = b1.size
    typ = np.tile(np.int32([0, 1, 3]), (n, 1))
    dt = np.tile([1.0, 1.0, 0.0], (n, 1))
    amp = np.stack([np.zeros(n), b1 * GAMMA / (2 * np.pi), np.zeros(n)], axis=1)
    freq = np.stack([np.zeros(n), np.full(n, 3.5 * 42.5764 * B0), np.zeros(n)], axis=1)
    ev = SimEvent(typ, dt, amp, np.zeros((n, 3)), freq, np.tile(np.int32([-1, -1, 0]), (n, 1)))
    grid = {"cest_k": np.geomspace(10.0, 5000.0, 64), "cest_f": np.geomspace(1e-5, 0.02, 32),
            "water_r1": 1.0 / np.linspace(0.8, 2.5, 16), "rel_b1": np.linspace(0.7, 1.3, 32)}
    return p, ev, initial_state(p), 4, grid


def run_dictionary(args, rank, world, local_rank):
    """Dictionary entries/s through the public API (mrf.generate_dictionary, host fingerprints out),
    then a 1% random subset of the entries against the float64 C oracle."""
    import torch
    from bmc_b200 import settings
    from bmc_b200.mrf import build_param_grid, generate_dictionary
    from bmc_b200.simulation import pack_params
    sys.path.insert(0, str(ROOT / "oracle"))
    import bmc_oracle as O
    torch.cuda.set_device(local_rank)
    p, ev, m0, mz, grid = dictionary_model()
    settings.use_precision(args.precision)
    try:
        generate_dictionary(p, ev, m0, {k: v[:2] for k, v in grid.items()}, mz)      # warm-up
        torch.cuda.synchronize()
        times = []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            entries, fp = generate_dictionary(p, ev, m0, grid, mz, chunk_size=262144)
            times.append(time.perf_counter() - t0)
    finally:
        settings.use_precision("f64")
    n = fp.shape[0]
    s = float(np.median(times))
    rng = np.random.default_rng(31)
    pick = np.sort(rng.choice(n, max(1, n // 100), replace=False))
    pb = build_param_grid(p, grid)
    from bmc_b200.simulation import SimParams
    sub = SimParams(*[np.asarray(v)[pick] for v in pb])
    t0 = time.perf_counter()
    want = O.c_simulate_z(pack_params(sub, pick.size), O.Events(*ev), np.broadcast_to(m0, (pick.size, m0.size)), 1, mz)
    cpu_s = time.perf_counter() - t0
    err = float(np.max(np.abs(fp[pick] - want)))
    return {"metric": "dictionary entries/s (MRF dictionary, public API)", "value": world * n / s,
            "unit": "entries/s", "n_gpus": world, "steps": len(times), "warmup": 1, "ms_per_step": s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
            "data": "synthetic grid", "config": {
                "workload": f"MRF dictionary: {n} entries (k 64 x f 32 x T1 16 x rel_b1 32) x 30 saturation rows, "
                            "water + amide + super-Lorentzian MT at 3 T, fingerprints to the host",
                "subset_checked": int(pick.size), "subset_max_abs_err_vs_float64_oracle": err,
                "cpu_oracle_entries_per_s": pick.size / cpu_s}}


def uneven_voxels(n, seed):
    """The uneven configuration: per voxel 1..5 CEST pools (2..6 pools with water), 41/61/81/121 offsets in
    -6..6 ppm at each of four B1 rungs (0.5, 1, 2, 4 uT), a train of 1..40 block pulses (50 ms, 5 ms gaps)
    per row, then the readout; k, f of every pool, water T2 and the B0 shift drawn in the batched
    configuration's ranges; water T1 1.3 s for every voxel (the shared value)."""
    from bmc_b200.fitting import Experiment
    from bmc_b200.simulation import SimEvent, SimParams, initial_state
    rng = np.random.default_rng(seed)
    tables = {}

    def table(n_off, n_p):
        key = (n_off, n_p)
        if key not in tables:
            ppm = np.linspace(-6.0, 6.0, n_off)
            rows = [(b, p) for b in (0.5, 1.0, 2.0, 4.0) for p in ppm]
            m, ne = len(rows), 2 * n_p + 1
            tables[key] = SimEvent(np.tile(np.int32([1, 0] * n_p + [3]), (m, 1)),
                                   np.tile([0.05, 0.005] * n_p + [0.0], (m, 1)),
                                   np.array([[b * GAMMA / (2 * np.pi), 0.0] * n_p + [0.0] for b, _ in rows]),
                                   np.zeros((m, ne)),
                                   np.array([[p * 42.5764 * B0, 0.0] * n_p + [0.0] for _, p in rows]),
                                   np.tile(np.int32([-1] * (ne - 1) + [0]), (m, 1)))
        return tables[key]

    exps = []
    for _ in range(n):
        nc = int(rng.integers(1, 6))
        pools = POOLS[:nc]
        p = SimParams(water_r1=np.float64(1 / 1.3), water_r2=np.float64(1 / rng.uniform(0.03, 0.12)),
                      water_f=np.float64(1.0), cest_k=rng.uniform(10.0, 5000.0, nc),
                      cest_f=rng.uniform(1e-5, 0.02, nc), cest_dw=np.array([q[0] for q in pools]),
                      cest_r1=np.array([1 / q[1] for q in pools]), cest_r2=np.array([1 / q[2] for q in pools]),
                      mt_k=np.float64(0.0), mt_f=np.float64(0.0), mt_dw=np.float64(0.0), mt_r1=np.float64(0.0),
                      mt_r2=np.float64(1.0), mt_lineshape=np.int64(0), b0=np.float64(B0),
                      gamma=np.float64(GAMMA), b0_inhom=np.float64(rng.uniform(-0.3, 0.3)), rel_b1=np.float64(1.0))
        ev = table(int(rng.choice([41, 61, 81, 121])), int(rng.integers(1, 41)))
        exps.append(Experiment(p, ev, initial_state(p), 2 * (1 + nc)))
    return exps, len(tables)


def run_uneven(args, rank, world, local_rank):
    """Fitted voxels/s of the uneven joint fit: every voxel its own pool count, offsets and pulse train;
    6 free values per voxel (k, f of the first two pools where they exist, water R2, B0 shift) and water
    R1 shared by every voxel; Gaussian noise sigma 0.005; 30 joint LM iterations from a fixed start
    (fit_joint_uneven: public API, host Z in, host values out)."""
    import torch
    from bmc_b200.fitting import FitSpec, FreeParam
    from bmc_b200.uneven import UnevenBatch, fit_joint_uneven
    torch.cuda.set_device(local_rank)
    n = args.voxels
    exps, n_tables = uneven_voxels(n, rank_seed(rank))
    spec = FitSpec([FreeParam("k1", "cest_k", 0, 100.0, 5.0, 6000.0, 300.0),
                    FreeParam("f1", "cest_f", 0, 1e-3, 1e-6, 0.05, 5e-4),
                    FreeParam("k2", "cest_k", 1, 100.0, 5.0, 6000.0, 300.0),
                    FreeParam("f2", "cest_f", 1, 1e-3, 1e-6, 0.05, 5e-4),
                    FreeParam("r2w", "water_r2", None, 10.0, 5.0, 50.0, 1 / 0.07),
                    FreeParam("b0", "b0_inhom", None, 0.1, -0.5, 0.5, 0.0),
                    FreeParam("r1w", "water_r1", None, 1.0, 0.2, 2.0, 0.7, scope="shared")])
    from bmc_b200.autotune import tune_dense_switch
    t0 = time.perf_counter()
    batch = UnevenBatch(exps)
    z_true = batch.simulate()
    rng = np.random.default_rng(rank_seed(rank) + 1)
    z = [zt + 0.005 * rng.standard_normal(zt.shape) for zt in z_true]
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tuning = tune_dense_switch(batch)
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    res = fit_joint_uneven(batch, spec, z, n_iter=30)
    torch.cuda.synchronize()
    fit_s = time.perf_counter() - t0
    chains = sum(g.n_chains for g in batch.groups)
    ev = sum(int(np.shape(e.events.dt)[0]) * int(np.shape(e.events.dt)[1]) for e in exps)
    nc = np.array([len(np.atleast_1d(e.params.cest_k)) for e in exps])
    return {"metric": "fitted voxels/s (uneven joint fit, shared water T1)", "value": world * n / fit_s,
            "unit": "voxels/s", "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": fit_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded), Gaussian noise sigma 0.005",
            "config": {"workload": f"uneven joint fit: {n} voxels, 2..6 pools, 41/61/81/121 offsets x 4 B1 rungs, "
                                   "1..40 block pulses per row, 6 free per voxel + shared water R1, 30 iterations",
                       "voxels_per_pool_count": {int(k): int((nc == k).sum()) for k in range(1, 6)},
                       "tables": n_tables, "chains": chains, "chain_events": ev, "setup_s": setup_s,
                       "autotune_s": tune_s,
                       "dense_switch": {k: v["dense_switch"] for k, v in tuning.items()},
                       "shared_r1w": {"fit": res.shared, "truth": 1 / 1.3,
                                      "rel_err": abs(res.shared * 1.3 - 1.0)},
                       "rms_over_sigma_median": float(np.median(res.rms / 0.005)),
                       "cost_first_last": [float(res.cost[0]), float(res.cost[-1])]}}


def lm_tangent_roofline(exp, spec, X_phys, peak):
    """The LM's tangent pass as the fit runs it (every free parameter's derivative at every offset) on
    `X_phys`, timed with CUDA events on the launching stream, against the kernels' own counts of the work
    they executed, in both tangent modes. The automatic mode (what bmc_lm_fit runs) takes the adjoint
    kernel on a single-event table such as the CW ladder: one launch, the exponential and its Frechet
    derivative in the readout's direction as a pair (dual) -- FLOPs per squaring 6 N^2 (N + 1), per Horner
    column product two operator products and a rank-one update -- then every tangent by a contraction
    (not counted: one sparse row per lane and tangent). Forward mode carries each tangent through a launch
    of its own as dual numbers: each primal multiply-add becomes 1 + 2 T (T tangents per launch), so a
    launch's FLOPs are its counted primal FLOPs times (1 + 2 T)."""
    import ctypes as C
    import torch
    from bmc_b200 import _lib, settings
    from bmc_b200.fitting import write_params, field_row
    from bmc_b200.simulation import DeviceEvents, pack_params, problem, tile_params, n_cest_of, state_size
    n = X_phys.shape[0]
    nc = n_cest_of(exp.params)
    N = state_size(nc)
    P = spec.n
    p = write_params(tile_params(exp.params, n), spec.to_scaled(X_phys), spec)
    dev_ev = DeviceEvents(exp.events)
    dP = torch.as_tensor(pack_params(p, n)).cuda()
    dM = torch.as_tensor(np.broadcast_to(np.asarray(exp.m0, np.float64), (n, N)).copy()).cuda()
    z = torch.empty((n, dev_ev.n_offsets), dtype=torch.float64, device="cuda")
    jz = torch.empty((P, n, dev_ev.n_offsets), dtype=torch.float64, device="cuda")
    seed = torch.as_tensor(np.tile(spec.scales[:, None], (1, n))).cuda()
    tg = _lib.Tangents()
    tg.n_tangents = P
    for i, sl in enumerate(spec.slots):
        tg.field_row[i] = field_row(sl.field, sl.index, nc)
    tg.d_seed, tg.d_dm0 = seed.data_ptr(), None
    pr = problem(n, dev_ev.n_offsets, dev_ev.n_events, nc, int(exp.mz_loc), _lib.F64)
    L = _lib.lib()
    stream = torch.cuda.current_stream()
    sh = C.c_void_p(stream.cuda_stream)
    call = lambda: _lib.check(L.bmc_simulate_jvp(pr, _lib.ptr(dP), dev_ev.struct, _lib.ptr(dM), None, tg,
                                                 _lib.ptr(z), _lib.ptr(jz), sh))
    nnz = 12 + 15 * nc
    flop_term = 2 * nnz + 2 * N
    T = 2 if nc <= 1 else 1                                  # forward mode's tangents per launch
    launches_fwd = (P + T - 1) // T
    out = {}
    for mode in ("auto", "forward"):
        settings.use_tangents(mode)
        try:
            call()
            work = torch.zeros(5, dtype=torch.int64, device="cuda")
            _lib.check(L.bmc_simulate_jvp_counted(pr, _lib.ptr(dP), dev_ev.struct, _lib.ptr(dM), None, tg,
                                                  _lib.ptr(z), _lib.ptr(jz), _lib.ptr(work), sh))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            e1.synchronize()
            out[mode] = ([int(x) for x in work.cpu()], e0.elapsed_time(e1))
        finally:
            settings.use_tangents("auto")
    (terms, hcols, squar, _, _), ms = out["auto"]
    (terms_f, hcols_f, squar_f, _, _), ms_f = out["forward"]
    flops_f = (terms_f * flop_term + hcols_f * flop_term + squar_f * 2.0 * N * N * (N + 1)) * (1 + 2 * T)
    adjoint = P > 1 and terms == 0 and squar_f == launches_fwd * squar
    if adjoint:
        flops = hcols * (2.0 * flop_term + 2 * N) + squar * 6.0 * N * N * (N + 1)
        kernel = f"adjoint_kernel<{nc}> (LM tangent pass: {P} tangents in 1 launch)"
    else:
        flops = flops_f
        kernel = f"chain_kernel<{nc}, double, {T}> (LM tangent pass, {launches_fwd} launches)"
    tf = flops / (ms * 1e-3) / 1e12
    tf_f = flops_f / (ms_f * 1e-3) / 1e12
    return {"bound": "fp64-fma", "achieved": tf, "peak": peak, "unit": "TFLOP/s",
            "frac": tf / peak if peak else None, "traffic": None, "kernel": kernel,
            "voxels": n, "offsets": dev_ev.n_offsets, "ms": ms, "flops": flops, "taylor_terms": terms,
            "dense_columns": hcols, "dense_squarings": squar,
            "forward_mode": {"ms": ms_f, "launches": launches_fwd, "flops": flops_f, "achieved": tf_f,
                             "frac": tf_f / peak if peak else None,
                             "kernel": f"chain_kernel<{nc}, double, {T}>"},
            "peak_source": "the forward leg's FP64 FMA probe of this run (burst)"}


def _oracle_lm_worker(job):
    """One voxel's plain LM on the float64 oracle for `n_iter` iterations (a spawn-pool worker)."""
    sys.path[:0] = [str(ROOT / "bmc-jax_b200"), str(ROOT / "oracle")]
    import bmc_oracle as O
    p, ev, m0, slots, z, x0, lo, hi, n_iter = job
    p, ev = O.Params(*p), O.Events(*ev)
    slots = [O.Slot(*s) for s in slots]
    t = time.perf_counter()
    O.fit_voxel(p, ev, m0, slots, z, x0, lo, hi, n_iter=n_iter)
    return time.perf_counter() - t


def fit_cpu_baseline(exp, spec, X_true, z, frac_plain, n_iter=30, sample_iters=3):
    """Plain LM on the float64 NumPy oracle (oracle.fit_voxel: the reference's LM schedule, exact
    forward-mode Jacobian, scipy expm per event), one voxel per host core in a spawn pool, timed for
    `sample_iters` iterations and extrapolated to n_iter (every iteration costs the same: one Jacobian and
    one trial residual); fitted voxels/s = cores x fraction within 1% (the GPU plain LM's, the same
    algorithm) / seconds per voxel."""
    import multiprocessing as mp
    cores = max(1, min(os.cpu_count() or 1, 32, len(z)))
    p = tuple(np.asarray(v, np.float64) for v in exp.params)
    ev = tuple(np.asarray(a) for a in exp.events)
    slots = [(s.field, s.index, s.scale) for s in spec.slots]
    m0 = np.asarray(exp.m0, np.float64)
    jobs = [(p, ev, m0, slots, z[i], spec.x0_phys, spec.lo_phys, spec.hi_phys, sample_iters) for i in range(cores)]
    # one BLAS thread per worker process (the workers inherit the environment at spawn)
    keys = ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")
    saved = {k: os.environ.get(k) for k in keys}
    os.environ.update({k: "1" for k in keys})
    try:
        with mp.get_context("spawn").Pool(cores) as pool:
            t0 = time.perf_counter()
            secs = pool.map(_oracle_lm_worker, jobs)
            wall = time.perf_counter() - t0
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    per_voxel = float(np.mean(secs)) * n_iter / sample_iters
    return {"value": cores * frac_plain / per_voxel, "unit": "voxels/s", "cores": cores, "kind": "port",
            "sample": f"{cores} voxels (one per process), {sample_iters} of {n_iter} plain LM iterations each "
                      f"({float(np.mean(secs)):.1f} s, {wall:.1f} s wall), float64 NumPy oracle "
                      f"(oracle/bmc_oracle.py fit_voxel); extrapolated to {n_iter} iterations and scaled by the "
                      f"fraction within 1% ({frac_plain:.3f})"}


def warm_vs_plain(args, rank, local_rank, peak_fp64=None):
    """Fitted voxels/s at <=1% parameter error, NN-warm vs plain LM: train the warm-start network on
    `--train` simulated ladders (noise sigma 0.005), then fit `--fit-voxels` held-out noise-free voxels
    (a) plainly, 30 iterations from the fixed x0, and (b) from the network's x0 with `--warm-iters`
    iterations plus the plain refit of every voxel whose warm fit ends above the rms threshold (keeping
    the better of the two). Both timed end to end through the public API (fitting.fit,
    LadderWarmStart.fit), host buffers in and out."""
    import torch
    from bmc_b200.fitting import fit
    from bmc_b200.warmstart import LadderWarmStart
    torch.cuda.set_device(local_rank)
    exp, spec, ranges = warm_model(args.pools)
    names = [s.name for s in spec.slots]
    seed = rank_seed(rank)
    ws = LadderWarmStart(exp, spec, ranges=ranges, sigma=0.005, seed=seed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Z, T, _ = ws.training_set(args.train, seed=seed)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    hist = ws.train(epochs=args.epochs, batch=4096, lr=1e-3, seed=seed, data=(Z, T))
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del Z, T
    torch.cuda.empty_cache()

    n = args.fit_voxels
    X_true = ws.draw(n, seed + 7919)
    z = ws.simulate64(X_true)
    # warm-up of both paths on a small slice (library load, workspaces, kernel attributes)
    fit(exp, spec, z[:256], n_iter=2)
    ws.fit(z[:256], n_iter_warm=2, n_iter_plain=2, fallback_rms=1e-4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain = fit(exp, spec, z, n_iter=30)
    plain_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    warm = ws.fit(z, n_iter_warm=args.warm_iters, n_iter_plain=30, fallback_rms=1e-4)
    warm_s = time.perf_counter() - t0
    ok_p = within_1pct(plain.x, X_true, names)
    ok_w = within_1pct(warm.x, X_true, names)
    x0_err = np.median(np.abs(warm.x0 / X_true - 1.0), axis=0)
    v_w = ok_w.sum() / warm_s
    v_p = ok_p.sum() / plain_s
    # the threshold rule against the literal judge (plain LM on every voxel, lower rms kept): how many
    # voxels keep a warm fit whose rms is above their plain fit's, and how many of those are not within 1%
    above = warm.rms > plain.rms * (1 + 1e-9) + 1e-15
    out = {"workload": f"warm-started LM: {n} voxels, water + {args.pools} CEST pools"
                       f"{' + MT' if args.pools >= 3 else ''}, ladder 4 x 61 CW (2 s), "
                       f"{spec.n} free ({', '.join(names)}); noise-free held-out voxels, parameters uniform in "
                       "the training ranges",
           "warm_fitted_voxels_per_s": v_w, "plain_fitted_voxels_per_s": v_p,
           "warm_over_plain": v_w / v_p if v_p else None, "unit": "voxels/s",
           "fraction_within_1pct": {"warm": float(ok_w.mean()), "plain": float(ok_p.mean())},
           "within_1pct_rule": "every free parameter within 1% of its truth (the B0 shift within 0.003 ppm)",
           "seconds": {"plain_lm": plain_s, "warm_total": warm_s,
                       **{f"warm_{k}": v for k, v in warm.seconds.items()}},
           "warm_iters": args.warm_iters, "plain_iters": 30, "refit_fraction": float(warm.refit.mean()),
           "judge": {"rule": "threshold: plain refit where the warm rms ends above 1e-4 (the better fit kept)",
                     "warm_rms_above_plain_fraction": float(above.mean()),
                     "of_those_not_within_1pct": int((above & ~ok_w).sum())},
           "median_x0_rel_err": dict(zip(names, map(float, x0_err))),
           "training": {"spectra": args.train, "epochs": args.epochs, "batch": 4096, "lr": 1e-3,
                        "simulate_s": gen_s, "train_s": train_s, "loss_first_last": [hist[0], hist[-1]],
                        "noise_sigma": 0.005},
           "mlp_roofline": mlp_roofline(ws.n_points, spec.n)}
    if peak_fp64 is None:
        peak_fp64 = fp64_peak()
    out["roofline"] = lm_tangent_roofline(exp, spec, X_true, peak_fp64)
    if not args.no_cpu:
        out["cpu_baseline"] = fit_cpu_baseline(exp, spec, X_true, z, float(ok_p.mean()))
    return out


def fma_peak(precision):
    """FMA throughput of this GPU now on the FP64 (precision F64) or FP32 pipe (TFLOP/s, best of three
    probe launches of 8 blocks per SM)."""
    import ctypes as C
    import torch
    from bmc_b200 import _lib
    stream = torch.cuda.current_stream()
    fl = C.c_double(0.0)
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(_lib.lib().bmc_probe_fma_peak(precision, sms * 8, 4096, C.byref(fl),
                                                 C.c_void_p(stream.cuda_stream)))
        e1.record(stream)
        e1.synchronize()
        best = max(best, fl.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    return best


def fp64_peak():
    """FP64 FMA throughput of this GPU now (TFLOP/s)."""
    from bmc_b200 import _lib
    return fma_peak(_lib.F64)


def run_lmtangent(args, rank, world, local_rank):
    """The LM tangent pass of the warm-start model (water + 4 CEST pools + MT, the 4 x 61 CW ladder, 6
    tangents) at --voxels voxels of seeded parameters: its own line, for profiling that kernel."""
    import torch
    torch.cuda.set_device(local_rank)
    exp, spec, ranges = warm_model(args.pools)
    lo, hi = np.array([a for a, _ in ranges]), np.array([b for _, b in ranges])
    X = lo + (hi - lo) * np.random.default_rng(rank_seed(rank)).random((args.voxels, spec.n))
    r = lm_tangent_roofline(exp, spec, X, fp64_peak())
    return {"metric": "LM tangent pass (Z and 6 tangents of the warm-start model)", "value": args.voxels / (r["ms"] * 1e-3),
            "unit": "voxels/s", "n_gpus": world, "steps": 1, "warmup": 1, "ms_per_step": r["ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": {"workload": f"LM tangent pass, {args.voxels} voxels"},
            "roofline": r}


def run_mlp(args, rank, world, local_rank):
    """The warm-start network's tcgen05 GEMMs alone (mlp_roofline on the five-pool ladder's shape,
    244 -> 3 x 256 -> 6): training steps at batch 4,096 replayed from a CUDA graph, --steps of them."""
    import torch
    torch.cuda.set_device(local_rank)
    r = mlp_roofline(244, 6, steps=max(1, args.steps))
    return {"metric": "warm-start network training step", "value": r["train_step_ms"], "unit": "ms",
            "n_gpus": world, "steps": max(1, args.steps), "warmup": 1, "ms_per_step": r["train_step_ms"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
            "data": "synthetic (random network and batch)",
            "config": {"workload": "MLP 244 -> 3 x 256 (GELU) -> 6, batch 4096, Adam"}, "roofline": r}


def run_warmfit(args, rank, world, local_rank):
    """The warm-vs-plain fit (warm_vs_plain) as its own bench line."""
    r = warm_vs_plain(args, rank, local_rank)
    return {"metric": "fitted voxels/s at <=1% param err, NN-warm vs plain LM", "value": world * r["warm_fitted_voxels_per_s"],
            "unit": "voxels/s", "n_gpus": world, "steps": 1, "warmup": 1,
            "ms_per_step": r["seconds"]["warm_total"] * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 LM, bf16/fp32 MLP",
            "data": "synthetic (seeded): parameters uniform in the ranges, noise-free held-out voxels",
            "config": {k: v for k, v in r.items() if k not in ("roofline", "cpu_baseline", "mlp_roofline")},
            "roofline": r["roofline"], "mlp_roofline": r["mlp_roofline"],
            **({"cpu_baseline": r["cpu_baseline"]} if "cpu_baseline" in r else {})}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["forward", "fit", "warmfit", "lmtangent", "dictionary", "uneven", "mlp",
                                           "phantom08", "phantom09", "phantom10", "phantom11"],
                    default="forward")
    ap.add_argument("--train", type=int, default=2_000_000, help="warmfit: simulated training spectra")
    ap.add_argument("--epochs", type=int, default=10, help="warmfit: training epochs")
    ap.add_argument("--warm-iters", type=int, default=8, help="warmfit: LM iterations from the network's x0")
    ap.add_argument("--spread-nodes", type=int, default=0, help="forward: B0-spread isochromats per voxel")
    ap.add_argument("--voxels", type=int, default=65536)
    ap.add_argument("--fit-voxels", type=int, default=65536, help="warm-vs-plain fit: held-out voxels")
    ap.add_argument("--no-fit", action="store_true", help="forward: leave out the warm-vs-plain fit leg")
    ap.add_argument("--offsets", type=int, default=101)
    ap.add_argument("--pulses", type=int, default=20)
    ap.add_argument("--pools", type=int, default=4, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--precision", choices=["f64", "mixed", "f32"], default="mixed")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    if args.workload.startswith("phantom"):
        if rank == 0:
            print(json.dumps(run_phantom(args)), flush=True)
        return
    run = {"fit": run_fit, "warmfit": run_warmfit, "lmtangent": run_lmtangent, "dictionary": run_dictionary,
           "uneven": run_uneven, "mlp": run_mlp}.get(args.workload, run_ours)
    line = run(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
