"""Benchmark of the fused FP32 CLE on the telegraph + capture workload.

Workload (one bench "step" = one whole simulate run): G=10 bursty genes with mixed
regulation, 20,000 cells per GPU, dt=0.01 h, T=50 h (5,000 Euler-Maruyama steps),
capture to an int32 count matrix.  Work unit: one cell-gene-step; one step is
20,000 x 10 x 5,000 = 1.0e9 units per GPU.

  value      device-resident throughput (network tables already on the GPU), CUDA events
             on the library's stream around each run; L2 flushed between runs.
  e2e        the same runs through the public host API: every step uploads the network from
             host arrays, runs, and copies readout + counts + efficiencies back to host
             (pooled page-locked arrays), timed on the host clock; the bytes are the
             library's own transfer counters.
  roofline   the register path's three algorithmic bounds per cell-gene-step (special-function
             ops, FP32 ops, integer ops of the Philox stream) against peaks measured live by
             the library's microkernels; the bound is the largest of the three.
  moment_err the largest per-gene mean / variance / Fano error (src/validate.jl:70-77
             convention) of the GPU run against the FP64 CPU oracle on the same increments,
             at the workload's full size.
  fp64_plain the plain FP64 one-kernel-per-step GPU CLE on the same workload.
  cpu_baseline  the FP64 CPU oracle (a port of the reference's cle.jl) on the whole workload,
             all host threads (the same run gives moment_err).
  readme / dense / batch / serve  the other workloads at N=1: the reference's published
             timing workload (CLE and binomial tau-leap, host wall clock per call), dense
             regulation on the tensor-core path, 256 uneven networks in one batch call, and the
             request server.

--impl reference times that CPU restatement alone (the Julia reference cannot run here).
--gpus N without a torchrun environment starts N ranks itself.  Multi-GPU: cells are
sharded by global index (weak scaling, no collective on the data path); the elapsed time
is the max over ranks; per-gene moment sums are all-reduced once after the timed region.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import socket
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CELLS_PER_GPU = 20000
L2_FLUSH_BYTES = 256 << 20
# algorithmic work per cell-gene-step of the register path, Hill exponent 2
SFU_PER_UNIT = 7            # Hill rcp, 2 sqrt, log + sin + cos of Box-Muller counted as 4 for two normals
FP32_BASE_PER_UNIT = 24     # Hill, M and P updates, Box-Muller, telegraph (+ 2 per in-edge / term source)
PHILOX_CALLS_PER_UNIT = 0.5  # two normals per cell-gene-step, four per Philox4x32-10 block
INT_OPS_PER_PHILOX = 80     # 10 rounds x (2 mul.lo + 2 mul.hi + 4 xor)


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="telegraph", choices=["telegraph", "readme", "dense", "batch", "serve"],
                    help="telegraph: the headline line (with the other workloads as extra keys at N=1); "
                         "dense / batch / serve: that workload alone")
    ap.add_argument("--requests", type=int, default=60, help="serve: number of requests")
    ap.add_argument("--rate", type=float, default=50.0, help="serve: Poisson arrival rate (1/s)")
    ap.add_argument("--batch-networks", type=int, default=256, help="batch: number of networks")
    ap.add_argument("--dense-steps", type=int, default=200, help="dense: Euler steps per timed run")
    ap.add_argument("--ref-sample-steps", type=int, default=250)
    ap.add_argument("--cpu-sample-cells", type=int, default=20000)
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-API leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle leg (cpu_baseline, moment_err)")
    ap.add_argument("--no-extra", action="store_true", help="skip the dense / batch / serve keys")
    return ap.parse_args()


def _dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def spawn_ranks(n: int, script: str = __file__, argv=None) -> int:
    """Run `script` (this file by default, with this call's arguments) under
    torch.distributed.run, one rank per GPU; returns the launcher's exit status."""
    argv = sys.argv[1:] if argv is None else list(argv)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", os.path.abspath(script)] + argv
    return subprocess.call(cmd)


def check_world(gpus: int, world: int):
    """The number of ranks running must be the number of GPUs asked for."""
    if world != gpus:
        raise SystemExit(f"bench.py: --gpus {gpus} but {world} rank(s) are running")


def max_over_ranks(x: float, world: int, device="cpu") -> float:
    """Maximum of x over the process group (x itself for one rank)."""
    if world == 1:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons while the GPU is busy."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period_ms=50):
        self.index = index
        self.period_ms = period_ms
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", str(self.period_ms)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

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
    """DRAM bytes per launch of the lane kernel from the committed ncu summary, if any."""
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


def _measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d.get("bf16_tflops_sustained", d["bf16_tflops"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


def _fp32_per_unit(net) -> float:
    """24 + 2 per additive in-edge + 2 per cooperative / redundant source, averaged over genes."""
    import numpy as np
    A = np.asarray(net.interactions) * np.asarray(net.basals)[:, None]
    np.fill_diagonal(A, 0.0)
    n_add = int(np.count_nonzero(A))
    n_src = sum(len(e.sources) for e in list(net.cooperative) + list(net.redundant))
    return FP32_BASE_PER_UNIT + 2.0 * (n_add + n_src) / net.G


def roofline_terms(units, kernel_s, fp32_per_unit, peaks):
    """The three algorithmic bounds of the register path; `peaks` = (fma/s, sfu/s, philox calls/s)."""
    fma_s, sfu_s, philox_s = peaks
    int_peak = philox_s * INT_OPS_PER_PHILOX
    counts = {"sfu": SFU_PER_UNIT, "fp32": fp32_per_unit, "int": PHILOX_CALLS_PER_UNIT * INT_OPS_PER_PHILOX}
    peak = {"sfu": sfu_s, "fp32": fma_s, "int": int_peak}
    src = {"sfu": "rsqrt.approx microkernel, 148 SMs", "fp32": "FFMA microkernel, 148 SMs",
           "int": "Philox4x32-10 microkernel (calls/s x 80 integer ops), round keys from parameters"}
    terms = {}
    for k in counts:
        achieved = counts[k] * units / kernel_s
        terms[k] = {"ops_per_unit": counts[k], "achieved_gops": achieved / 1e9, "peak_gops": peak[k] / 1e9,
                    "frac": achieved / peak[k], "ps_per_unit_at_peak": 1e12 * counts[k] / peak[k],
                    "peak_source": "measured live: " + src[k]}
    bound = max(terms, key=lambda k: terms[k]["ps_per_unit_at_peak"])
    return bound, terms


def cpu_oracle_run(wl, cells, steps, threads, seed):
    """FP64 CPU restatement of cle.jl on `cells` x `steps` of the workload: (units/s, s, result)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    t0 = time.perf_counter()
    out = oracle.simulate(wl.net, wl.kin, dt=wl.dt, cell_num=cells, n_steps=steps, seed=seed, nthreads=threads)
    el = time.perf_counter() - t0
    return cells * wl.net.G * steps / el, el, out


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
        cpu_oracle_run(wl, max(cells // 10, 100), max(steps // 10, 10), threads, 123)
    els = []
    for _ in range(args.steps):
        _, el, _ = cpu_oracle_run(wl, cells, steps, threads, 123)
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


def _event_ms(fn, stream):
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_ours(args):
    rank, world, local = _dist()
    check_world(args.gpus, world)
    import numpy as np
    import torch
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    wl = pkg.config1()
    N = CELLS_PER_GPU
    G = wl.net.G
    n_steps = pkg.n_steps(wl.T, wl.dt)
    units = N * G * n_steps
    seed = 2024

    ctx = pkg.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    run = pkg.DeviceRun(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, T=wl.T, readout=wl.readout, seed=seed,
                        capture=wl.capture, cell_offset=rank * N, ctx=ctx)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    clocks = ClockSampler(local).start()
    time.sleep(0.5)  # nvidia-smi's first sample comes a few hundred ms after it starts
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            run.launch()
    barrier()
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
    clk = clocks.stop()
    launches = ctx.launches - launches0
    per = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(per), world, f"cuda:{local}")
    value = units * world * args.steps / (total_ms * 1e-3)
    kernel_ms = statistics.mean(per)  # one fused launch per non-population run

    # the per-gene moment sums of all ranks' cells, all-reduced once (FP64) after the timed region
    from scrna_b200 import sharding
    allreduce = None
    if world > 1:
        tot = sharding.allreduce_moments(sharding.moment_sums(run.read()[0]))
        allreduce = {"backend": "nccl", "doubles": int(tot.size), "cells": int(round(tot[0, 0]))}

    # roofline: the register path's three bounds, peaks measured live by the library
    fma_s, sfu_s, _ = pkg.measure_pipe_peaks(ctx)
    philox_s = pkg.measure_philox_rate(ctx)
    bound, terms = roofline_terms(units, kernel_ms * 1e-3, _fp32_per_unit(wl.net), (fma_s, sfu_s, philox_s))
    roof = {"bound": bound, "achieved": terms[bound]["achieved_gops"], "peak": terms[bound]["peak_gops"],
            "unit": "Gop/s", "frac": terms[bound]["frac"], "traffic": _traffic_per_launch(),
            "kernel_ms": kernel_ms, "terms": terms,
            "note": "bound = the term with the longest time per cell-gene-step at its measured peak"}

    # FP64 plain one-kernel-per-step baseline on the same workload
    fp64 = None
    if not args.no_fp64:
        run64 = pkg.DeviceRun(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, T=wl.T, readout=wl.readout,
                              seed=seed, capture=wl.capture, precision="fp64_plain", cell_offset=rank * N,
                              ctx=ctx)
        with torch.cuda.stream(stream):
            run64.launch()
            torch.cuda.synchronize()
            reps = 2
            ms64 = _event_ms(lambda: [run64.launch() for _ in range(reps)], stream) / reps
        fp64 = {"value": units / (ms64 * 1e-3), "ms_per_step": ms64, "unit": "cell·gene·steps/s",
                "launches_per_step": n_steps + 4}
        run64.close()

    # e2e through the public host API: network upload, run, results to host, every step
    e2e = None
    if not args.no_e2e:
        e2e_steps = max(3, min(args.steps, 10))

        def e2e_step():
            h = pkg.NetHandle(wl.net, ctx)
            out = pkg.simulate(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, T=wl.T, readout=wl.readout,
                               seed=seed, capture=wl.capture, cell_offset=rank * N, ctx=ctx, handle=h)
            h.close()
            return out

        e2e_step()
        barrier()
        b0 = ctx.transfer_bytes()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            e2e_step()
        e2e_s = max_over_ranks(time.perf_counter() - t0, world, f"cuda:{local}")
        b1 = ctx.transfer_bytes()
        e2e = {"value": units * world * e2e_steps / e2e_s, "unit": "cell·gene·steps/s",
               "h2d_bytes_per_step": (b1[0] - b0[0]) // e2e_steps, "d2h_bytes_per_step": (b1[1] - b0[1]) // e2e_steps,
               "note": "per step: network upload from host arrays, run, readout + counts + efficiencies to host"}
        barrier()

    # CPU oracle on the whole workload: the CPU baseline and the moment-error check in one run
    cpu = moment = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        Xg = pkg.simulate(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, T=wl.T, readout="both", seed=seed, ctx=ctx)
        rate, el, ref = cpu_oracle_run(wl, N, n_steps, threads, seed)
        Xr = np.hstack([ref["M"].T, ref["P"].T])
        errs = pkg.moment_errors(Xg, Xr)
        cpu = {"value": rate, "unit": "cell·gene·steps/s", "cores": threads, "kind": "port",
               "sample": f"the whole workload: {N} cells x {n_steps} Euler steps x {G} genes ({el:.1f} s)"}
        moment = {"max": max(float(v.max()) for v in errs.values()),
                  **{k: float(v.max()) for k, v in errs.items()},
                  "against": "FP64 CPU oracle, same Philox increments, mRNA and protein of every gene",
                  "convention": "|a-b|/max(|a|,|b|,1e-10) (src/validate.jl:70-77)"}

    extra = {}
    if rank == 0 and world == 1 and not args.no_extra:
        for name, fn in (("readme", leg_readme), ("dense", leg_dense), ("batch", leg_batch), ("serve", leg_serve)):
            try:
                extra[name] = fn(pkg, args, local)
            except Exception as e:  # a failed leg is reported, never silently dropped
                extra[name] = {"error": f"{type(e).__name__}: {e}"}

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
            "moment_err": moment,
            "roofline": roof,
            "fp64_plain": fp64,
            "speedup_vs_fp64_plain": (value / world) / fp64["value"] if fp64 else None,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        if allreduce:
            line["moment_allreduce"] = allreduce
        line.update(extra)
        print(json.dumps(line), flush=True)
    run.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def leg_dense(pkg, args, device):
    """Dense regulation, G=2000, 65,536 cells, dt=0.005: the fused tcgen05 path, per Euler step."""
    import torch
    wl = pkg.config2()
    ctx = pkg.Context(device)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    steps = args.dense_steps
    G, N = wl.net.G, wl.cell_num
    run = pkg.DeviceRun(wl.net, pkg.CLE(wl.dt), wl.kin, cell_num=N, T=0.0, n_steps=steps, readout="protein",
                        seed=7, ctx=ctx)
    run.launch()
    torch.cuda.synchronize()
    clocks = ClockSampler(device).start()
    el = [_event_ms(run.launch, stream) * 1e-3 for _ in range(3)]
    clk = clocks.stop()
    per = sum(el) / len(el)
    units = G * N * steps
    K = G + len(wl.net.cooperative) + len(wl.net.redundant)  # gene columns + one column per term
    flops = 2.0 * G * K * N * steps
    algo_bytes = 18.0 * units  # M, P read + write (FP32), 16-bit activations written
    pk = _measured_peaks()
    out = {"workload": wl.name, "value": units / per, "unit": "cell·gene·steps/s", "ms_per_euler_step": 1e3 * per / steps,
           "euler_steps": steps, "gemm_tflops": flops / per / 1e12,
           "tensor_frac_of_sustained": flops / per / 1e12 / pk["bf16_tflops_sustained"],
           "hbm_gbs_algorithmic": algo_bytes / per / 1e9, "hbm_frac": algo_bytes / per / 1e9 / pk["hbm_gbs"],
           "bound_frac": max(flops / per / 1e12 / pk["bf16_tflops_sustained"], algo_bytes / per / 1e9 / pk["hbm_gbs"]),
           "peaks_source": pk["source"], "dtype": "bf16 contraction inputs, f32 state", "clocks": clk}
    run.close()
    ctx.close()
    return out


def leg_batch(pkg, args, device):
    """256 networks, G ~ LogUniform(5, 500), cells ~ LogUniform(1k, 50k), half with a Moran population,
    dt=0.01, T=50: one simulate_gpu_batch call (persistent launches per kernel group)."""
    import torch
    wls = pkg.config3(n_networks=args.batch_networks)
    nets = [w.net for w in wls]
    cells = [w.cell_num for w in wls]
    pops = [w.population for w in wls]
    units = sum(w.net.G * w.cell_num * pkg.n_steps(w.T, w.dt) for w in wls)
    ctx = pkg.Context(device)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    call = lambda: pkg.simulate_gpu_batch(nets, pkg.CLE(0.01), wls[0].kin, cell_num=cells, T=50.0,
                                          populations=pops, seed=1, ctx=ctx)
    t0 = time.perf_counter()
    call()
    first = time.perf_counter() - t0
    clocks = ClockSampler(device).start()
    t0 = time.perf_counter()
    dev_ms = _event_ms(call, stream)
    host_s = time.perf_counter() - t0
    clk = clocks.stop()
    ctx.close()
    return {"workload": f"batch-{len(wls)}-uneven", "value": units / (dev_ms * 1e-3), "unit": "cell·gene·steps/s",
            "e2e_value": units / host_s, "s_per_call_device": dev_ms * 1e-3, "s_per_call_host": host_s,
            "first_call_s": first, "units_per_call": units,
            "networks_with_population": sum(p is not None for p in pops),
            "note": "device: CUDA events on the call's stream (results copied to host inside); "
                    "e2e: host clock around the whole call", "clocks": clk}


def leg_serve(pkg, args, device):
    """Poisson request stream (rate --rate), G ~ LogUniform(5, 500), cells ~ LogUniform(1k, 100k),
    T ~ U(20, 60) h, bursty / constitutive mix, capture on: continuous-batching server."""
    import threading
    import numpy as np
    reqs = pkg.config4_requests(n_requests=args.requests, rate_per_s=args.rate)
    ctx = pkg.Context(device)
    handles = [pkg.NetHandle(w.net, ctx) for _, w in reqs]
    srv = pkg.Server(ctx, chunk_steps=500)
    tickets = [None] * len(reqs)
    clocks = ClockSampler(device, period_ms=200).start()
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
    clk = clocks.stop()
    st = srv.stats()
    srv.close()
    ctx.close()
    units = st["units_done"]
    offered = sum(w.net.G * w.cell_num * pkg.n_steps(w.T, w.dt) for _, w in reqs) / reqs[-1][0]
    return {"workload": "serve-poisson", "requests": len(reqs), "rate_per_s": args.rate,
            "value": units / makespan, "unit": "cell·gene·steps/s",
            "p50_latency_s": float(np.percentile(lats, 50)), "p99_latency_s": float(np.percentile(lats, 99)),
            "makespan_s": makespan, "busy_s": st["busy_s"], "offered_load": offered,
            "sustainable_rate_per_s": (len(reqs) / st["busy_s"]) if st["busy_s"] > 0 else None,
            "chunks": st["chunks"], "clocks": clk}


def leg_readme(pkg, args, device):
    """The workload of the reference's published timing table (README.md:68-80, the 5-gene case
    of experiments/validate_analytical.jl:184-232): 5 unregulated genes with basals 1..5, k_t=1,
    mu_m=0.1, mu_p=0.2, 5,000 cells, dt=0.1, T=300 (3,000 steps), protein readout.  Each call is
    timed on the host clock around simulate (upload, run, copy back), after one warm-up call,
    as the reference times it (that call also pays the autotuner's one measurement for the
    new shape), then once more on the same shape (`s_per_call_repeat`); errors are against
    the exact two-stage moments."""
    import numpy as np
    ctx = pkg.Context(device)
    net = pkg.GeneNetwork(5, [1.0, 2.0, 3.0, 4.0, 5.0], np.zeros((5, 5)))
    k_t, mu_m, mu_p = 1.0, 0.1, 0.2
    kin = pkg.KineticParams(k_t=k_t, K_d=50.0, n=2.0, mu_m=mu_m, mu_p=mu_p)
    beta = np.arange(1.0, 6.0)
    p_mean = k_t * beta / (mu_m * mu_p)
    p_var = p_mean * (1.0 + k_t / (mu_m + mu_p))
    units = 5 * 5000 * 3000
    out = {"workload": "readme-G5-N5000-T300-dt0.1", "units_per_call": units,
           "reference_rtx5060_s": {"CLE": 0.22, "BinomialTauLeap": 0.45}}
    for name, alg in (("CLE", pkg.CLE(0.1)), ("BinomialTauLeap", pkg.BinomialTauLeap(0.1))):
        pkg.simulate(net, alg, kin, cell_num=100, T=10.0, readout="protein", seed=1, ctx=ctx)
        t0 = time.perf_counter()
        Y = pkg.simulate(net, alg, kin, cell_num=5000, T=300.0, readout="protein", seed=42, ctx=ctx)
        el = time.perf_counter() - t0
        t0 = time.perf_counter()
        pkg.simulate(net, alg, kin, cell_num=5000, T=300.0, readout="protein", seed=43, ctx=ctx)
        el2 = time.perf_counter() - t0
        out[name] = {"s_per_call": el, "value": units / el, "unit": "cell·gene·steps/s",
                     "s_per_call_repeat": el2, "value_repeat": units / el2,
                     "max_mean_err": float(np.max(np.abs(Y.mean(0) - p_mean) / p_mean)),
                     "max_var_err": float(np.max(np.abs(Y.var(0, ddof=1) - p_var) / p_var))}
    ctx.close()
    return out


def run_single_leg(args):
    import json as _json
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    fn = {"readme": leg_readme, "dense": leg_dense, "batch": leg_batch, "serve": leg_serve}[args.workload]
    print(_json.dumps(fn(pkg, args, 0)), flush=True)


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload != "telegraph":
        run_single_leg(args)
    elif args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
