"""Benchmark of the fused FP32 CLE on the telegraph + capture workload.

Workload (one bench "step" = one whole simulate run): G=10 bursty genes with mixed
regulation, 20,000 cells per GPU, dt=0.01 h, T=50 h (5,000 Euler-Maruyama steps),
capture to an int32 count matrix.  Work unit: one cell-gene-step; one step is
20,000 x 10 x 5,000 = 1.0e9 units per GPU.

  value      device-resident throughput (network tables already on the GPU), CUDA events
             on the library's stream around each run; L2 flushed between runs.
  e2e        the same runs through the public host API (scrna_cle_simulate via
             simulate(...)): network upload from host arrays, run, readout + counts +
             efficiencies copied back to host, timed on the host clock.
  roofline   special-function-unit (MUFU) issue bound of the register path: the
             algorithmic 7 SFU operations per cell-gene-step against the SFU throughput
             measured live by the library's microkernel.
  fp64_plain the plain FP64 one-kernel-per-step GPU CLE on the same workload.
  cpu_baseline  the FP64 CPU oracle (a port of the reference's cle.jl) on a bounded
             sample of the workload, all host threads.

--impl reference times that CPU restatement alone (the Julia reference cannot run here).
Multi-GPU (torchrun): cells are sharded by global index (weak scaling, no collective on
the data path); the elapsed time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SFU_PER_UNIT = 7          # algorithmic special-function ops per cell-gene-step (n = 2)
CELLS_PER_GPU = 20000
L2_FLUSH_BYTES = 256 << 20


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="telegraph", choices=["telegraph", "dense", "batch", "serve"],
                    help="telegraph: the headline workload; the others are reported in DESIGN.md")
    ap.add_argument("--requests", type=int, default=60, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=50.0, help="serve: Poisson arrival rate (1/s)")
    ap.add_argument("--batch-networks", type=int, default=256, help="batch: number of networks")
    ap.add_argument("--dense-steps", type=int, default=0,
                    help="dense: Euler steps per run (default: the workload's T/dt = 8,000)")
    ap.add_argument("--cpu-sample-cells", type=int, default=20000)
    ap.add_argument("--cpu-sample-steps", type=int, default=1000)
    ap.add_argument("--ref-sample-steps", type=int, default=250)
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-API leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    return ap.parse_args()


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
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
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _traffic_per_launch():
    """DRAM bytes per launch of the fused kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "cle_warpcell_telegraph_capture_G10_N20000.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def cpu_reference(pkg, wl, cells, steps, threads):
    """FP64 CPU restatement of cle.jl on `cells` x `steps` of the workload; returns units/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    t0 = time.perf_counter()
    oracle.simulate(wl.net, wl.kin, dt=wl.dt, cell_num=cells, n_steps=steps, seed=123, nthreads=threads)
    el = time.perf_counter() - t0
    return cells * wl.net.G * steps / el, el


def run_reference(args):
    rank, world, _ = _dist()
    if rank != 0:
        return
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    wl = pkg.config1()
    threads = os.cpu_count() or 1
    cells, steps = args.cpu_sample_cells, args.ref_sample_steps
    for _ in range(max(args.warmup, 0)):
        cpu_reference(pkg, wl, max(cells // 10, 100), max(steps // 10, 10), threads)
    rates, els = [], []
    for _ in range(args.steps):
        r, el = cpu_reference(pkg, wl, cells, steps, threads)
        rates.append(r)
        els.append(el)
    total_units = cells * wl.net.G * steps * args.steps
    value = total_units / sum(els)
    line = {
        "impl": "reference", "metric": "cell_gene_steps_per_s", "value": value, "unit": "cell·gene·steps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(els) / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "genes": wl.net.G, "cells": cells, "euler_steps": steps,
                   "dt": wl.dt, "note": "bounded sample of the telegraph+capture workload"},
        "cpu_baseline": {"value": value, "unit": "cell·gene·steps/s", "cores": threads, "kind": "port",
                         "sample": f"{cells} cells x {steps} Euler steps x {wl.net.G} genes per step"},
        "e2e": {"value": value, "unit": "cell·gene·steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    rank, world, local = _dist()
    import numpy as np
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    wl = pkg.config1()
    N = CELLS_PER_GPU
    G = wl.net.G
    n_steps = pkg.n_steps(wl.T, wl.dt)
    units = N * G * n_steps

    ctx = pkg.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    run = pkg.DeviceRun(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, T=wl.T, readout=wl.readout, seed=2024,
                        capture=wl.capture, cell_offset=rank * N, ctx=ctx)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            run.launch()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = ctx.launches
    evs = []
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run.launch()
            e1.record(stream)
            evs.append((e0, e1))
    barrier()
    launches = ctx.launches - launches0
    per = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(per)
    if world > 1:
        t = torch.tensor([total_ms], device=f"cuda:{local}", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    clk = clocks.stop()
    value = units * world * args.steps / (total_ms * 1e-3)
    kernel_ms = statistics.mean(per)  # one fused launch per non-population run

    # roofline: SFU issue bound, peak measured live by the library's microkernel
    fma_s, sfu_s, int_s = pkg.measure_pipe_peaks(ctx)
    achieved_sfu = SFU_PER_UNIT * units / (kernel_ms * 1e-3)
    traffic = _traffic_per_launch()

    # FP64 plain one-kernel-per-step baseline on the same workload
    fp64 = None
    if not args.no_fp64:
        run64 = pkg.DeviceRun(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, T=wl.T, readout=wl.readout,
                              seed=2024, capture=wl.capture, precision="fp64_plain", cell_offset=rank * N,
                              ctx=ctx)
        with torch.cuda.stream(stream):
            run64.launch()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            reps = 2
            e0.record(stream)
            for _ in range(reps):
                run64.launch()
            e1.record(stream)
        torch.cuda.synchronize()
        ms64 = e0.elapsed_time(e1) / reps
        fp64 = {"value": units / (ms64 * 1e-3), "ms_per_step": ms64, "unit": "cell·gene·steps/s",
                "launches_per_step": n_steps + 4}
        run64.close()

    # e2e through the public host API (host arrays in, host arrays out)
    e2e_steps = 0 if args.no_e2e else max(3, min(args.steps, 10))
    h2d = d2h = 0
    t0 = time.perf_counter()
    for i in range(1 + e2e_steps if e2e_steps else 0):
        if i == 1:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
        X, counts, eff = pkg.simulate(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, T=wl.T, readout=wl.readout,
                                      seed=2024, capture=wl.capture, cell_offset=rank * N, ctx=ctx)
        d2h = X.nbytes + counts.nbytes + eff.nbytes
    e2e_s = time.perf_counter() - t0
    net = wl.net
    h2d = (net.basals.nbytes + net.interactions.nbytes + net.k_on.nbytes + net.k_off.nbytes
           + 16 * (len(net.cooperative) + len(net.redundant)) + 48 * G)
    e2e_value = units * world * e2e_steps / e2e_s if e2e_steps else None

    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        cpu_rate, cpu_el = cpu_reference(pkg, wl, args.cpu_sample_cells, args.cpu_sample_steps, threads)
        cpu = {"value": cpu_rate, "unit": "cell·gene·steps/s", "cores": threads, "kind": "port",
               "sample": f"{args.cpu_sample_cells} cells x {args.cpu_sample_steps} Euler steps x {G} genes "
                         f"({cpu_el:.1f} s)"}

    if rank == 0:
        line = {
            "metric": "cell_gene_steps_per_s", "value": value, "unit": "cell·gene·steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": wl.name, "genes": G, "cells_per_gpu": N, "euler_steps_per_run": n_steps,
                       "dt": wl.dt, "T": wl.T, "telegraph": True, "capture": "lognormal-binomial int32",
                       "units_per_step": units * world, "l2": "flushed (256 MB write) between timed runs",
                       "parallelism": f"cells sharded over {world} GPU(s)"},
            "roofline": {"bound": "sfu", "achieved": achieved_sfu / 1e9, "peak": sfu_s / 1e9,
                         "unit": "Gop/s (MUFU)", "frac": achieved_sfu / sfu_s, "traffic": traffic,
                         "kernel_ms": kernel_ms, "algorithmic_sfu_per_unit": SFU_PER_UNIT,
                         "peak_source": "measured live (rsqrt.approx microkernel, 148 SMs)",
                         "fp32_fma_peak_gops": fma_s / 1e9, "int_peak_gops": int_s / 1e9},
            "fp64_plain": fp64,
            "speedup_vs_fp64_plain": (value / world) / fp64["value"] if fp64 else None,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell·gene·steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    run.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def _event_time(fn, stream):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1e-3


def run_dense(args):
    """Dense regulation, G=2000, 65,536 cells, dt=0.005, T=40 (8,000 steps): tensor-core path."""
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    wl = pkg.config2()
    ctx = pkg.Context(0)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    n_steps = args.dense_steps if args.dense_steps > 0 else pkg.n_steps(wl.T, wl.dt)
    G, N = wl.net.G, wl.cell_num
    run = pkg.DeviceRun(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, T=0.0, n_steps=n_steps, readout="protein",
                        seed=7, ctx=ctx)
    run.launch()
    torch.cuda.synchronize()
    el = [_event_time(run.launch, stream) for _ in range(max(1, args.steps))]
    per = sum(el) / len(el)
    units = G * N * n_steps
    K = G + len(wl.net.cooperative) + len(wl.net.redundant)  # gene columns + one column per term
    flops = 2.0 * G * K * N * n_steps
    algo_bytes = 18.0 * units  # M, P read + write (FP32), 16-bit activations written
    peaks = _measured_peaks()
    line = {"workload": wl.name, "value": units / per, "unit": "cell·gene·steps/s", "s_per_run": per,
            "euler_steps": n_steps, "gemm_tflops": flops / per / 1e12, "tensor_frac": flops / per / 1e12 / peaks["bf16_tflops"],
            "hbm_gbs_algorithmic": algo_bytes / per / 1e9, "hbm_frac": algo_bytes / per / 1e9 / peaks["hbm_gbs"],
            "peaks": peaks}
    print(json.dumps(line), flush=True)


def _measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def run_batch_workload(args):
    """256 networks, G ~ LogUniform(5, 500), cells ~ LogUniform(1k, 50k), half with a Moran
    population, dt=0.01, T=50: one simulate_gpu_batch call (persistent launches per group)."""
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    wls = pkg.config3(n_networks=args.batch_networks)
    nets = [w.net for w in wls]
    cells = [w.cell_num for w in wls]
    pops = [w.population for w in wls]
    units = sum(w.net.G * w.cell_num * pkg.n_steps(w.T, w.dt) for w in wls)
    kin = wls[0].kin
    t0 = time.perf_counter()
    pkg.simulate_gpu_batch(nets, pkg.CLE(0.01), kin, cell_num=cells, T=50.0, populations=pops, seed=1)
    warm = time.perf_counter() - t0
    els = []
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        pkg.simulate_gpu_batch(nets, pkg.CLE(0.01), kin, cell_num=cells, T=50.0, populations=pops, seed=1)
        els.append(time.perf_counter() - t0)
    per = sum(els) / len(els)
    print(json.dumps({"workload": "batch-%d-uneven" % len(wls), "value": units / per, "unit": "cell·gene·steps/s",
                      "s_per_run": per, "first_run_s": warm, "units_per_run": units,
                      "networks_with_population": sum(p is not None for p in pops),
                      "note": "host wall clock around the whole batch call, results copied to host"}), flush=True)


def run_serve(args):
    """Poisson request stream (rate --rate), G ~ LogUniform(5, 500), cells ~ LogUniform(1k, 100k),
    T ~ U(20, 60) h, bursty / constitutive mix, capture on: continuous-batching server."""
    import threading
    import numpy as np
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    reqs = pkg.config4_requests(n_requests=args.requests, rate_per_s=args.rate)
    ctx = pkg.default_context()
    handles = [pkg.NetHandle(w.net, ctx) for _, w in reqs]
    srv = pkg.Server(ctx, chunk_steps=500)
    tickets = [None] * len(reqs)
    t_start = time.perf_counter()

    def submitter():
        for i, (t_arr, w) in enumerate(reqs):
            delay = t_start + t_arr - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            tickets[i] = srv.submit(handles[i], pkg.CLE(w.dt), w.kin, cell_num=w.cell_num, T=w.T,
                                    readout="mrna", seed=i, capture=w.capture)

    th = threading.Thread(target=submitter)
    th.start()
    lats = []
    for i in range(len(reqs)):
        while tickets[i] is None:
            time.sleep(0.001)
        lats.append(srv.wait(tickets[i], -1)[3])
    th.join()
    makespan = time.perf_counter() - t_start
    st = srv.stats()
    srv.close()
    units = st["units_done"]
    offered = sum(w.net.G * w.cell_num * pkg.n_steps(w.T, w.dt) for _, w in reqs) / reqs[-1][0]
    print(json.dumps({"workload": "serve-poisson", "requests": len(reqs), "rate_per_s": args.rate,
                      "value": units / makespan, "unit": "cell·gene·steps/s", "p50_latency_s": float(np.percentile(lats, 50)),
                      "p99_latency_s": float(np.percentile(lats, 99)), "makespan_s": makespan,
                      "busy_s": st["busy_s"], "offered_load": offered,
                      "max_stable_rate_per_s": (units / st["busy_s"]) / (units / len(reqs)) if st["busy_s"] > 0 else None,
                      "chunks": st["chunks"]}), flush=True)


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "dense":
        run_dense(args)
    elif args.workload == "batch":
        run_batch_workload(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
