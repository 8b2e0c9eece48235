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


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except (OSError, ValueError):
        return {}


# ------------------------------------------------------------------------------------------------
# CPU baseline: the C oracle on the host cores, bounded sample
# ------------------------------------------------------------------------------------------------
def cpu_baseline(P, M0, ev, n_cest, budget_s=15.0, kind="port"):
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
    O.c_simulate_z(P[:, :n_vox], events, M0[:n_vox], n_cest, mz, threads)
    el = time.perf_counter() - t
    return {"value": n_vox / el, "unit": "Z-spectra/s", "cores": threads, "kind": kind,
            "sample": f"{n_vox} voxels x {n_off} offsets x {ev[0].shape[1]} events, float64 Pade-13 "
                      f"expm per event (oracle/bmc_oracle.c, OpenMP), {el:.1f} s"}


# ------------------------------------------------------------------------------------------------
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
    prec = _lib.F32 if args.precision == "f32" else _lib.F64

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

    def step(params=dP, m0=dM, evs=dev_ev, out=dZ):
        _lib.check(L.bmc_simulate(pr, C.c_void_p(params.data_ptr()), evs.struct, C.c_void_p(m0.data_ptr()), None,
                                  C.c_void_p(out.data_ptr()), sh))

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # 256 MB > L2 (126 MB)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)

    # executed work of one launch (deterministic), from the kernel's own counters
    work = torch.zeros(4, dtype=torch.int64, device=dev)
    _lib.check(L.bmc_simulate_counted(pr, C.c_void_p(dP.data_ptr()), dev_ev.struct, C.c_void_p(dM.data_ptr()),
                                      None, C.c_void_p(dZ.data_ptr()), C.c_void_p(work.data_ptr()), sh))
    torch.cuda.synchronize(dev)
    terms, hcols, squar, executed = [int(x) for x in work.cpu()]
    nnz = 12 + 15 * nc                                   # nonzeros of A (+ C folded into term 1)
    flop_term = 2 * nnz + 2 * N                          # operator product + scaling + accumulation
    NA = N + 1
    flops = terms * flop_term + hcols * flop_term + squar * 2.0 * N * N * NA

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

    # end to end: host buffers in, Z back to the host, copies inside the timed region
    e2e = []
    for _ in range(args.steps):
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

    # FMA peak of this GPU, measured now (burst, like a kernel timed alone)
    fl = C.c_double(0.0)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(L.bmc_probe_fma_peak(prec, sms * 8, 4096, C.byref(fl), sh))
        e1.record(stream)
        e1.synchronize()
        best = max(best, fl.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)

    achieved = flops / (ms * 1e-3) / 1e12
    value = world * nv / (ms * 1e-3)
    line = {
        "metric": "Z-spectra/s (batched forward simulation)", "value": value, "unit": "Z-spectra/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == _lib.F64 else "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"forward simulation: {nv} voxels per GPU x {n_off} offsets x {n_ev} events, "
                               f"water + {nc} CEST pools + super-Lorentzian MT (state {N}, augmented {NA}), "
                               f"20 Gaussian 50 ms pulses + 5 ms gaps, spoiler, 3 s recovery, ADC",
                   "voxels_per_gpu": nv, "offsets": n_off, "events": n_ev, "pools": nc,
                   "parallelism": f"dp{world} (voxels sharded, no collective)",
                   "l2": "flushed between timed steps (256 MB write, untimed)"},
        "e2e": {"value": world * nv / (e2e_ms * 1e-3), "unit": "Z-spectra/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "roofline": {"bound": "fp64-fma" if prec == _lib.F64 else "fp32-fma", "achieved": achieved,
                     "peak": best, "unit": "TFLOP/s", "frac": achieved / best if best else None,
                     "traffic": None, "kernel": "chain_kernel",
                     "flops_per_launch": flops, "taylor_terms": terms, "taylor_terms_executed": executed,
                     "dense_columns": hcols,
                     "dense_squarings": squar,
                     "peak_source": "measured in this run: FMA-chain probe kernel (bmc_probe_fma_peak), burst"},
        "clocks": clocks,
        "gpu_launches": 2 * args.steps,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(P, M0, ev, nc, budget_s=args.cpu_budget)
    return line


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


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--voxels", type=int, default=65536)
    ap.add_argument("--offsets", type=int, default=101)
    ap.add_argument("--pulses", type=int, default=20)
    ap.add_argument("--pools", type=int, default=4, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--precision", choices=["f64", "f32"], default="f64")
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
    line = run_ours(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
