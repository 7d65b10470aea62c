"""Benchmark of the routed FP16 SpMM hot path (one JSON line on rank 0).

Workload: the large routed SpMM — SBM graph, N = 200,000 nodes, mean degree
50 (~10.2 M nnz with self loops), 2,000 communities of ~100 nodes, 70 % of
edges inside a community, power-law degrees, nodes randomly permuted, GCN
values in FP16; B = 200,000 x 128 FP16 ~ N(0,1).  Seeded synthetic data: the
reference ships no datasets.

A step = one routed forward C = A . B (FP16 in, FP32 accumulate, FP32 out,
the reference's output type) over the whole matrix with the device plan
resident in HBM.  Between timed steps a 256 MiB buffer is written to flush
L2 (126 MB); each step is timed alone with CUDA events on its stream.

  value       SpMM TFLOP/s = 2 * nnz * K / t, summed over ranks (replicas)
  e2e         same metric through the public API with host buffers: per step
              the H2D copy of B from pinned memory, the routed kernel and the
              D2H copy of C into pinned memory
  roofline    routed kernel vs measured HBM copy bandwidth, algorithmic bytes
              nnz*(4+2) + (M+1)*4 + N*K*2 + M*K*4 per launch
  cpu_baseline / --impl reference: the oracle's C restatement of the SpMM
              (FP16 operands, FP32 accumulation, OpenMP on all host cores)

Multi-GPU: the path does not shard (replicas only); under torchrun every rank
runs the full workload independently and rank 0 reports max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tr-spmm_b200"))
sys.path.insert(0, ROOT)

WORKLOAD = "large_routed"
METRIC = "SpMM TFLOP/s, %HBM roofline; fwd+bwd ms vs plain CSR on one B200 at FP16 tol"
UNIT = "TFLOP/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic():
    """Per-launch DRAM bytes of the routed kernel from the committed ncu
    summary (profiles/routed_kernel_large_routed.txt, line 'traffic_bytes_per_launch: N')."""
    path = os.path.join(ROOT, "profiles", "routed_kernel_large_routed.txt")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi SM clock / throttle samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def algorithmic_bytes(nnz, m, n_cols, k, out_bytes=4):
    return nnz * (4 + 2) + (m + 1) * 4 + n_cols * k * 2 + m * k * out_bytes


def cpu_baseline(g, b, budget_s=12.0):
    """Oracle C SpMM (FP16 operands, FP32 accumulation) on all host cores,
    repeated for ~budget_s seconds; TFLOP/s."""
    import oracle
    vals = g.values.astype(np.float16)
    out = np.empty((g.n_rows, b.shape[1]), dtype=np.float32)
    threads = oracle.max_threads()
    oracle.spmm_f16_f32(g.indptr, g.indices, vals, b, threads=threads, out=out)   # warm-up
    reps, t0 = 0, time.perf_counter()
    while True:
        oracle.spmm_f16_f32(g.indptr, g.indices, vals, b, threads=threads, out=out)
        reps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or reps >= 50:
            break
    tflops = 2.0 * g.nnz * b.shape[1] * reps / el / 1e12
    return {"value": tflops, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"full workload ({g.nnz} nnz x K={b.shape[1]}), {reps} passes in {el:.1f} s"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    from trspmm import graphs
    g, b = graphs.make_workload(WORKLOAD)
    import oracle
    vals = g.values.astype(np.float16)
    out = np.empty((g.n_rows, b.shape[1]), dtype=np.float32)
    threads = oracle.max_threads()
    for _ in range(max(1, args.warmup)):
        oracle.spmm_f16_f32(g.indptr, g.indices, vals, b, threads=threads, out=out)
    steps = max(1, min(args.steps, 20))      # a CPU pass takes ~0.1-1 s; bounded sample
    t0 = time.perf_counter()
    for _ in range(steps):
        oracle.spmm_f16_f32(g.indptr, g.indices, vals, b, threads=threads, out=out)
    el = time.perf_counter() - t0
    v = 2.0 * g.nnz * b.shape[1] * steps / el / 1e12
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "ms_per_step": el / steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_nodes": g.n_rows, "nnz": g.nnz, "k": int(b.shape[1]),
                       "out": "f32"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"full workload, {steps} passes"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference has no CPU SpMM; its GPU operator's semantics are run by the "
                    "oracle's C restatement (C = A.B over the routed operand) on all host cores"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    import trspmm
    from trspmm import graphs

    world, rank, local = dist_setup()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", world_size=world, rank=rank,
                                timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    g, b = graphs.make_workload(WORKLOAD)
    k = int(b.shape[1])
    t0 = time.perf_counter()
    plan = trspmm.Plan.from_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    plan_s = time.perf_counter() - t0
    bd = torch.from_numpy(b).to(dev)
    cd = torch.empty((g.n_rows, k), dtype=torch.float32, device=dev)
    ip = torch.from_numpy(g.indptr).to(dev)
    ix = torch.from_numpy(g.indices).to(dev)
    iv = torch.from_numpy(g.values.astype(np.float16)).to(dev)
    c2 = torch.empty_like(cd)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for s, e in ev:
            flush.fill_(1.0)
            s.record(stream)
            fn()
            e.record(stream)
        torch.cuda.synchronize()
        return [s.elapsed_time(e) for s, e in ev]

    routed = lambda: plan.spmm(bd, out=cd)
    plain = lambda: trspmm.spmm_csr(ip, ix, iv, bd, g.n_rows, out=c2)

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        times = timed(routed, args.steps, max(3, args.warmup))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = float(np.mean(times))
    ms_t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    flops = 2.0 * g.nnz * k
    value = flops * world / (ms_max * 1e-3) / 1e12

    plain_times = timed(plain, min(args.steps, 500), 5)
    plain_ms = float(np.mean(plain_times))
    err_vs_plain = float((cd - c2).abs().max().item() / max(c2.abs().max().item(), 1e-30))

    # end to end through the public API with host buffers
    b_host = torch.from_numpy(b).pin_memory()
    c_host = torch.empty((g.n_rows, k), dtype=torch.float32).pin_memory()

    def e2e_step():
        bd.copy_(b_host, non_blocking=True)
        plan.spmm(bd, out=cd)
        c_host.copy_(cd, non_blocking=True)

    e2e_steps = max(3, min(args.steps, 50))
    for _ in range(3):
        e2e_step()
    torch.cuda.synchronize()
    s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_ev.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e_ev.record(stream)
    torch.cuda.synchronize()
    e2e_ms = s_ev.elapsed_time(e_ev) / e2e_steps
    e2e_t = torch.tensor([e2e_ms], device=dev)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_val = flops * world / (float(e2e_t.item()) * 1e-3) / 1e12

    peak, peak_kind = _peaks()
    abytes = algorithmic_bytes(g.nnz, g.n_rows, g.n_cols, k, 4)
    achieved = abytes / (ms * 1e-3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(g, b)
    clocks = clk.summary()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_nodes": g.n_rows, "nnz": g.nnz, "k": k,
                       "out": "f32", "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"replicas{world}", "plan": "exact routing, built once"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": _profile_traffic(),
                         "peak_kind": peak_kind, "algorithmic_bytes": abytes},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(b.nbytes),
                    "d2h_bytes_per_step": int(g.n_rows * k * 4)},
            "gpu_launches": args.steps,
            "clocks": clocks,
            "extra": {"plain_csr_ms": plain_ms,
                      "plain_csr_tflops": flops / (plain_ms * 1e-3) / 1e12,
                      "routed_vs_plain_csr": plain_ms / ms,
                      "routed_vs_plain_max_rel_diff": err_vs_plain,
                      "plan_build_s": plan_s, "plan": plan.info,
                      "e2e_ms_per_step": float(e2e_t.item())},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
