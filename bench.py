"""Benchmark of the routed FP16 SpMM hot path (one JSON line on rank 0).

Workload: the large routed SpMM — SBM graph, N = 200,000 nodes, mean degree
50 (~10.2 M nnz with self loops), 2,000 communities of ~100 nodes, 70 % of
edges inside a community, power-law degrees, nodes randomly permuted, GCN
values; B = 200,000 x 128 FP16 ~ N(0,1).  Seeded synthetic data: the
reference ships no datasets.

A step = one routed forward + adjoint, as a GNN layer's training step runs
it: C = A . B (routed forward plan), dB = A^T . dC (routed adjoint plan,
built once) and dval = SDDMM(dC, B) on A's pattern (the edge-weight
gradient), the last two in one fused pass over A^T where the plan allows;
FP16 operands, FP32 accumulation and outputs, dC a fixed synthetic FP16
gradient.  Plans are built once, outside the timed region, with the plan
options the autotuner (trspmm.autotune) finds fastest for this graph: for
the forward among the window engine's routings and the block engine
(tcgen05 over 128-row blocks of label-ordered rows), for the adjoint the
fastest whole backward.
Between timed steps a 256 MiB buffer is written to flush L2 (126 MB); each
step is timed alone with CUDA events on its stream.

  value       TFLOP/s = 3 * 2 * nnz * K / t (forward, adjoint, SDDMM), summed
              over ranks (replicas)
  e2e         same metric through the public API with host buffers: per
              step B and dC copied from pinned memory, the autograd forward and
              backward of trspmm.autograd.routed_spmm, and C, dB and dval copied
              back to pinned memory
  roofline    the dominant kernel against the measured HBM copy bandwidth:
              the fused backward (one launch: dB = A^T dC and dval) with
              algorithmic bytes per launch = nnz*(4+2+4+4) + (N+1)*4 + M*K*2
              + N*K*2 + N*K*4, or, when the forward's kernel is the longer
              one, the block-engine forward (or the window engine's CUDA-core
              residual pass) with nnz*(4+2) + (M+1)*4 + N*K*2 + M*K*4 (CSR
              bytes: the layout's padding and metadata count against it);
              extra.forward_roofline reports the forward either way
  cpu_baseline / --impl reference: the oracle's C restatement of the same
              step (FP16 operands, FP32 accumulation, OpenMP on all host cores);
              extra.cpu_torch_sparse_forward: the forward alone with
              torch.sparse CSR (FP32) on all host cores
  extra       the same step with the plain single-route CSR kernel (forward on
              A, adjoint on a CSR of A^T, same SDDMM), and like for like:
              the forward against the plain CSR kernel, the backward against
              the same fused pass over a natural-order CSR of A^T, and the
              step at equal fusion; per-pass times and the autotuner's tables

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


def _profile_traffic(name):
    """Per-launch DRAM bytes of a kernel from its committed ncu summary
    (profiles/<name>, line 'traffic_bytes_per_launch: N'); None when that
    summary is absent."""
    path = os.path.join(ROOT, "profiles", name)
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


def adjoint_sddmm_bytes(nnz, m, n, k, out_bytes=4, entry_ids=False):
    """Fused backward over A^T (n rows): per entry its column, value and dval
    (4+2+4 bytes; plus a 4-byte entry id when dval is stored through one);
    dC (m x k FP16) and B (n x k FP16) read once; dB (n x k) written once."""
    per = 4 + 2 + 4 + (4 if entry_ids else 0)
    return nnz * per + (n + 1) * 4 + m * k * 2 + n * k * 2 + n * k * out_bytes


def block_bwd_bytes(nnz, chunks, m, n, k, out_bytes=4, entry_ids=False):
    """Tensor-core backward over a block plan of A^T (n rows): per entry its
    packed value and position and its dval (4+4 bytes; plus a 4-byte entry id
    when dval is stored through one), per chunk its 16 columns and entry
    offset; dC (m x k FP16) and B (n x k FP16) read once; dB (n x k) written
    once."""
    per = 4 + 4 + (4 if entry_ids else 0)
    return nnz * per + chunks * (16 * 4 + 4) + m * k * 2 + n * k * 2 + n * k * out_bytes


def _single_stream(adj_opts):
    """Adjoint plans whose entries form one stream (block plans, all-residual
    window plans): the edges can be numbered in their entry order."""
    if adj_opts.get("engine", "window") == "block":
        return True
    return adj_opts.get("demote_below", 0) >= 1000


def step_bytes(nnz, m, n, k):
    """Forward + adjoint + SDDMM algorithmic bytes (FP32 outputs)."""
    sddmm = nnz * 4 + m * k * 2 + n * k * 2 + nnz * 4
    return algorithmic_bytes(nnz, m, n, k) + algorithmic_bytes(nnz, n, m, k) + sddmm


def router_comparison(g):
    """Seconds to route the graph (the reference's parameters, compat mode):
    the host router on all host threads, and the device router with the CSR
    already on the device (tables brought back to the host); both produce
    the same 29 tables."""
    import torch
    import trspmm
    host = trspmm.route(g.indptr, g.indices, g.values)
    d = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (g.indptr, g.indices, g.values)]
    trspmm.route_device(*d, out="torch")      # first call: module load, shared-memory limits
    t0 = time.perf_counter()
    dev = trspmm.route_device(*d, out="torch")
    torch.cuda.synchronize()
    dev_s = time.perf_counter() - t0
    same = all(np.array_equal(a, b.cpu().numpy().reshape(a.shape)) for a, b in zip(host[:29], dev[:29]))
    t0 = time.perf_counter()
    trspmm.route_device(*d)                   # the same with every table copied to the host
    dev_host_s = time.perf_counter() - t0
    return {"host": float(host[-1]), "device": float(dev[-1]), "device_api_s": dev_s,
            "device_with_host_copies_s": dev_host_s, "tables_equal": bool(same),
            "host_threads": os.cpu_count(),
            "note": "host: the host router on all threads, tables in host memory; device: "
                    "the device router, tables left on the device (the GPU kernels' input)"}


def transpose_csr(indptr, indices, values, n_rows, n_cols):
    import scipy.sparse as sp
    a = sp.csr_matrix((values, indices, indptr), shape=(n_rows, n_cols)).T.tocsr()
    a.sort_indices()
    return a.indptr.astype(np.int32), a.indices.astype(np.int32), a.data.astype(np.float32)


def torch_sparse_cpu_forward(g, b, reps=5):
    """C = A.B with torch.sparse CSR on all host cores (FP32: the CPU CSR
    matmul has no FP16 kernel): the stock CPU library baseline for the
    forward, reported beside the oracle's whole-step baseline.  Median of `reps` after one
    warm-up."""
    import torch
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")            # "beta state" notice of sparse CSR
        A = torch.sparse_csr_tensor(torch.from_numpy(g.indptr.astype(np.int64)),
                                    torch.from_numpy(g.indices.astype(np.int64)),
                                    torch.from_numpy(g.values.astype(np.float32)),
                                    size=(g.n_rows, g.n_cols), check_invariants=False)
    B = torch.from_numpy(np.asarray(b, dtype=np.float32))
    A @ B
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        A @ B
        ts.append(time.perf_counter() - t0)
    t = float(np.median(ts))
    return {"value": 2.0 * g.nnz * B.shape[1] / t / 1e12, "unit": UNIT, "cores": threads,
            "dtype": "f32", "op": "forward C = A.B, torch.sparse CSR", "ms": t * 1e3}


class CpuStep:
    """The step on the host cores with the oracle's C arithmetic (FP16
    operands, FP32 accumulation, OpenMP on every host thread)."""

    def __init__(self, g, gt, b, dc):
        import oracle
        self.oracle = oracle
        self.threads = oracle.max_threads()
        self.g, self.gt, self.b, self.dc = g, gt, b, dc
        self.v16, self.vt16 = g.values.astype(np.float16), gt[2].astype(np.float16)
        k = b.shape[1]
        self.c = np.empty((g.n_rows, k), dtype=np.float32)
        self.db = np.empty((g.n_cols, k), dtype=np.float32)
        self.dv = np.empty(g.nnz, dtype=np.float32)

    def __call__(self):
        o, g, gt, t = self.oracle, self.g, self.gt, self.threads
        o.spmm_f16_f32(g.indptr, g.indices, self.v16, self.b, threads=t, out=self.c)
        o.spmm_f16_f32(gt[0], gt[1], self.vt16, self.dc, threads=t, out=self.db)
        o.sddmm_f16_f32(g.indptr, g.indices, self.dc, self.b, threads=t, out=self.dv)

    def time(self, budget_s=12.0, max_steps=50):
        """(seconds per step, steps timed) over about budget_s seconds."""
        self()
        reps, t0 = 0, time.perf_counter()
        while True:
            self()
            reps += 1
            el = time.perf_counter() - t0
            if el >= budget_s or reps >= max_steps:
                return el / reps, reps


def batched_comparison(dev, flush, n_graphs=512, k=64, reps=20):
    """The batched workload: 512 power-law graphs (20-500 nodes, degree
    4-32), forward (block engine) + fused backward at K=64.  One
    block-diagonal plan pair, the step captured in a CUDA graph, vs one plan
    pair per graph launched in a loop (eagerly from Python, and the same loop
    captured in a graph), with the same plan options."""
    import torch
    from trspmm import graphs
    from trspmm.batched import BatchedStep, PerGraphLoop
    g = graphs.batched(num_graphs=n_graphs)
    # block-engine forward (the small graphs' rows share columns within a
    # block), fused CUDA-core backward
    opts = dict(engine="block", promote_min=0, row_scale=True,
                adjoint_options={"demote_below": 1000})
    bs = BatchedStep(g, k, device=dev, **opts)
    loop = PerGraphLoop(g, k, device=dev, **opts)
    b = torch.from_numpy(graphs.dense_features(g.n_cols, k, seed=1)).to(dev)
    dc = torch.from_numpy(graphs.dense_features(g.n_rows, k, seed=2)).to(dev)
    for st in (bs, loop):
        st.b.copy_(b)
        st.dc.copy_(dc)

    def med(fn):
        for _ in range(3):
            fn()
        ts = []
        for _ in range(reps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    loop_eager = med(loop.run)
    bs.capture()
    batched_graph = med(bs.replay)
    loop.capture()
    loop_graph = med(loop.replay)
    return {"graphs": n_graphs, "nodes": g.n_rows, "nnz": g.nnz, "k": k,
            "batched_graph_ms": batched_graph, "per_graph_loop_ms": loop_eager,
            "per_graph_loop_captured_ms": loop_graph,
            "speedup_vs_loop": loop_eager / batched_graph,
            "speedup_vs_captured_loop": loop_graph / batched_graph}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(ms, world, device):
    """The largest of the ranks' per-step times (every rank calls this, in the
    same order; world 1 returns ms)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_tflops(flops_per_step, world, ms_max):
    """Whole-job throughput: every rank processes one step's units in ms_max."""
    return flops_per_step * world / (ms_max * 1e-3) / 1e12


def workload(name=WORKLOAD):
    from trspmm import graphs
    g, b = graphs.make_workload(name)
    dc = graphs.dense_features(g.n_rows, b.shape[1], "normal", seed=g.seed + 101)
    return g, b, dc


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    g, b, dc = workload(args.workload)
    gt = transpose_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    k = int(b.shape[1])
    step = CpuStep(g, gt, b, dc)
    for _ in range(max(1, min(args.warmup, 3))):
        step()
    steps = max(1, min(args.steps, 10))      # a CPU step takes ~1 s; bounded sample
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    el = time.perf_counter() - t0
    v = 3 * 2.0 * g.nnz * k * steps / el / 1e12
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "ms_per_step": el / steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16",
            "data": "synthetic",
            "config": {"workload": args.workload, "n_nodes": g.n_rows, "nnz": g.nnz, "k": k,
                       "step": "forward + adjoint + SDDMM", "out": "f32"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": step.threads, "kind": "port",
                             "sample": f"full workload, {steps} steps"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference has no CPU SpMM and no backward; its operator's semantics "
                    "(C = A.B over the routed operand) and the adjoint are run by the oracle's C "
                    "restatement on all host cores"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner and use the reference's routing (exact mode)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the 512-graph batched comparison reported under extra")
    ap.add_argument("--workload", default=WORKLOAD,
                    choices=["large_routed", "route_mix", "gcn_diff", "plain_small"],
                    help="graph of the step (default: the headline workload); the others "
                         "are for profiling the routes they exercise")
    ap.add_argument("--plan-options", default=None,
                    help="JSON plan options to use instead of the autotuner's choice "
                         '(e.g. \'{"demote_below": 1000}\'), for profiling runs')
    ap.add_argument("--adjoint-options", default=None,
                    help="JSON options of the adjoint plan (default: the autotuner's "
                         "backward choice, or --plan-options when given)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    import trspmm
    from trspmm import autotune
    from trspmm.autograd import RoutedAdjacency, routed_spmm

    world, rank, local = dist_setup()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", world_size=world, rank=rank,
                                timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    g, b, dc = workload(args.workload)
    k = int(b.shape[1])
    gt = transpose_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)

    # ---- plan options: the autotuner's choice for the forward plan ------------
    # and, for the adjoint plan, the fastest whole backward (dB and dval)
    t0 = time.perf_counter()
    bwd_report = {"results": []}
    if args.plan_options is not None:
        opts, tune_report = json.loads(args.plan_options), {"results": []}
        adj_opts = json.loads(args.adjoint_options) if args.adjoint_options else dict(opts)
    elif args.no_tune:
        opts, tune_report = {}, {"results": []}
        adj_opts = {}
    else:
        opts, tune_report = autotune.tune(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, k,
                                          device=dev, row_scale=True, reps=5)
        if args.adjoint_options:
            adj_opts = json.loads(args.adjoint_options)
        else:
            adj_opts, bwd_report = autotune.tune(g.indptr, g.indices, g.values, g.n_rows,
                                                 g.n_cols, k, device=dev, row_scale=True, reps=5,
                                                 backward=True)
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    # per-entry arrays (the values and dval) in the adjoint plan's entry order
    # where it has one, so that the backward stores dval sequentially
    edge_order = "adjoint" if _single_stream(adj_opts) else "csr"
    adj = RoutedAdjacency(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, device=dev,
                          row_scale=True, adjoint_options={"promote_min": 0, **adj_opts},
                          edge_order=edge_order, **{"promote_min": 0, **opts})
    plan_s = time.perf_counter() - t0
    pf, pa = adj.fwd, adj.adj

    bd = torch.from_numpy(b).to(dev)
    dcd = torch.from_numpy(dc).to(dev)
    cd = torch.empty((g.n_rows, k), dtype=torch.float32, device=dev)
    dbd = torch.empty((g.n_cols, k), dtype=torch.float32, device=dev)
    dvd = torch.empty(g.nnz, dtype=torch.float32, device=dev)
    ip, ix = adj.indptr, adj.indices
    iv = torch.from_numpy(g.values.astype(np.float16)).to(dev)
    ipt, ixt = torch.from_numpy(gt[0]).to(dev), torch.from_numpy(gt[1]).to(dev)
    ivt = torch.from_numpy(gt[2].astype(np.float16)).to(dev)
    c2, db2, dv2 = torch.empty_like(cd), torch.empty_like(dbd), torch.empty_like(dvd)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for s_, e_ in ev:
            flush.fill_(1.0)
            s_.record(stream)
            fn()
            e_.record(stream)
        torch.cuda.synchronize()
        return [s_.elapsed_time(e_) for s_, e_ in ev]

    def routed_step():
        pf.spmm(bd, out=cd)
        pa.adjoint_sddmm(ip, ix, dcd, bd, db=dbd, dval=dvd)

    def plain_step():
        trspmm.spmm_csr(ip, ix, iv, bd, g.n_rows, out=c2)
        trspmm.spmm_csr(ipt, ixt, ivt, dcd, g.n_cols, out=db2)
        trspmm.sddmm_csr(ip, ix, dcd, bd, out=dv2)

    warm = max(3, args.warmup)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        times = timed(routed_step, args.steps, warm)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = float(np.mean(times))
    ms_max = max_over_ranks(ms, world, dev)
    flops = 3 * 2.0 * g.nnz * k
    value = whole_job_tflops(flops, world, ms_max)

    # per-pass times and the plain single-route comparison (outside the timed region)
    n_side = min(args.steps, 100)
    fwd_ms = float(np.mean(timed(lambda: pf.spmm(bd, out=cd), n_side, 3)))
    adj_ms = float(np.mean(timed(lambda: pa.spmm(dcd, out=dbd), n_side, 3)))
    adj_sddmm_ms = float(np.mean(timed(lambda: pa.adjoint_sddmm(ip, ix, dcd, bd, db=dbd, dval=dvd),
                                       n_side, 3)))
    sddmm_ms = float(np.mean(timed(lambda: trspmm.sddmm_csr(ip, ix, dcd, bd, out=dvd), n_side, 3)))
    fwd_block = pf.info["engine"] == trspmm.TR_ENGINE_BLOCK
    if fwd_block:
        res_ms = None                  # the block engine has no CUDA-core residual pass
    else:
        res_mask = trspmm.TR_ROUTE_ALL | trspmm.TR_ROUTE_RESIDUAL_PASS
        res_ms = float(np.mean(timed(lambda: pf.spmm(bd, out=c2, route_mask=res_mask), n_side, 3)))
    plain_ms = float(np.mean(timed(plain_step, n_side, 3)))
    plain_fwd_ms = float(np.mean(timed(lambda: trspmm.spmm_csr(ip, ix, iv, bd, g.n_rows, out=c2),
                                       n_side, 3)))
    # like for like backward: the same fused dB + dval pass over a CSR of A^T
    # in natural order (no reordering, no tiles: the plain single route)
    plain_adj = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                                  transpose=True, row_scale=True, demote_below=1000)
    if adj.edge_id is not None:
        plain_adj.renumber_edges(adj.edge_id)     # dval in the same order as the routed arm
    plain_bwd_ms = float(np.mean(timed(
        lambda: plain_adj.adjoint_sddmm(ip, ix, dcd, bd, db=db2, dval=dv2), n_side, 3)))
    plain_adj.close()
    # the step's fused backward with the bitwise-repeatable combine
    det_bwd_ms = None
    if pa.info["engine"] == trspmm.TR_ENGINE_WINDOW:
        pa.set_deterministic(True)
        det_bwd_ms = float(np.mean(timed(
            lambda: pa.adjoint_sddmm(ip, ix, dcd, bd, db=db2, dval=dv2), n_side, 3)))
        pa.set_deterministic(False)
    # the other deterministic backward: the block plan of A^T with the
    # tensor-core backward (edges in its own entry order), unless it is the
    # step's own adjoint plan already
    block_bwd_ms = None
    if pa.info["engine"] != trspmm.TR_ENGINE_BLOCK and k in (64, 128):
        bplan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                                  transpose=True, row_scale=True, engine="block", reorder=True)
        border = bplan.entry_order(dev)
        bid = torch.empty_like(border)
        bid[border.long()] = torch.arange(g.nnz, dtype=torch.int32, device=dev)
        bplan.renumber_edges(bid)
        block_bwd_ms = float(np.mean(timed(
            lambda: bplan.adjoint_sddmm(ip, ix, dcd, bd, db=db2, dval=dv2), n_side, 3)))
        bplan.close()
        del border, bid
    # the same forward with the features in FP32 (FP32-feature route, CUDA
    # cores; a window plan, the block engine's FP32 kernel being a fallback)
    pf32 = pf if pf.info["engine"] == trspmm.TR_ENGINE_WINDOW else trspmm.Plan.build(
        g.indptr, g.indices, g.values, g.n_rows, g.n_cols, row_scale=True, demote_below=1000)
    b32 = bd.float()
    c3 = torch.empty_like(cd)
    f32_ms = float(np.mean(timed(lambda: pf32.spmm(b32, out=c3), n_side, 3)))
    routed_step()
    plain_step()
    pf32.spmm(b32, out=c3)
    torch.cuda.synchronize()
    rel = lambda a_, b_: float((a_ - b_).abs().max().item() / max(b_.abs().max().item(), 1e-30))
    err = {"C": rel(cd, c2), "dB": rel(dbd, db2), "dval": rel(adj.to_csr_order(dvd), dv2)}
    fp32_route = {"ms": f32_ms, "tflops": 2.0 * g.nnz * k / (f32_ms * 1e-3) / 1e12,
                  "max_rel_diff_vs_fp16_features": rel(c3, cd)}
    del b32, c3

    # ---- end to end through the public API with host buffers -------------------
    # A training step through routed_spmm autograd: every step uploads its
    # B and its upstream gradient G (= dC) from pinned host memory, computes
    # C = A(w) B, the loss <C, G>, and the backward (dB, dw), and reads its
    # result back into pinned host memory: the loss and the squared norms of
    # dB and dw (three FP32 numbers; the gradients stay on the device for the
    # optimizer).  Beside it, the same step downloading all of C, dB and dw
    # (extra.e2e_full_outputs).  The loop is pipelined the way a training
    # loop over batches would be: step i+1's upload (copy stream s_in) and
    # step i's download (copy stream s_out) run while step i computes, in two
    # alternating device-input / host-output slots.  The timed region spans
    # the first upload to the last download.
    b_host = torch.from_numpy(b).pin_memory()
    dc_host = torch.from_numpy(dc).pin_memory()
    w_dev = adj.values.clone()                  # the adjacency's edge order
    c_host = [torch.empty((g.n_rows, k), dtype=torch.float32).pin_memory() for _ in range(2)]
    db_host = [torch.empty((g.n_cols, k), dtype=torch.float16).pin_memory() for _ in range(2)]
    dw_host = [torch.empty(g.nnz, dtype=torch.float32).pin_memory() for _ in range(2)]
    m_host = [torch.empty(3, dtype=torch.float32).pin_memory() for _ in range(2)]
    b_in = [torch.empty((g.n_cols, k), dtype=torch.float16, device=dev) for _ in range(2)]
    dc_in = [torch.empty((g.n_rows, k), dtype=torch.float16, device=dev) for _ in range(2)]
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    ev_in = [torch.cuda.Event() for _ in range(2)]      # slot's inputs uploaded
    ev_used = [torch.cuda.Event() for _ in range(2)]    # slot's step computed
    ev_out = [torch.cuda.Event() for _ in range(2)]     # slot's outputs downloaded

    def upload(i):
        sl = i % 2
        with torch.cuda.stream(s_in):
            s_in.wait_event(ev_used[sl])                # the slot's previous step is done with it
            b_in[sl].copy_(b_host, non_blocking=True)
            dc_in[sl].copy_(dc_host, non_blocking=True)
            ev_in[sl].record(s_in)

    def compute_and_download(i, full):
        sl = i % 2
        stream.wait_event(ev_in[sl])
        bb = b_in[sl].detach().requires_grad_(True)
        w = w_dev.detach().requires_grad_(True)
        c = routed_spmm(adj, bb, w)
        if full:
            c.backward(dc_in[sl])
            outs = (c.detach(), bb.grad, w.grad)
        else:
            loss = (c * dc_in[sl]).sum()                # d loss / dC = G
            loss.backward()
            outs = (torch.stack([loss.detach(), bb.grad.float().square().sum(),
                                 w.grad.square().sum()]),)
        ev_used[sl].record(stream)
        with torch.cuda.stream(s_out):
            s_out.wait_event(ev_used[sl])
            if full:
                c_host[sl].copy_(outs[0], non_blocking=True)
                db_host[sl].copy_(outs[1], non_blocking=True)
                dw_host[sl].copy_(outs[2], non_blocking=True)
            else:
                m_host[sl].copy_(outs[0], non_blocking=True)
            for t in outs:
                t.record_stream(s_out)                  # keep alive until downloaded
            ev_out[sl].record(s_out)

    def e2e_run(n, full):
        upload(0)
        for i in range(n):
            if i + 1 < n:
                upload(i + 1)
            compute_and_download(i, full)
        for sl in range(2):
            stream.wait_event(ev_out[sl])

    e2e_steps = max(3, min(args.steps, 30))

    def e2e_time(full):
        e2e_run(3, full)
        torch.cuda.synchronize()
        s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_ev.record(stream)
        s_in.wait_event(s_ev)
        e2e_run(e2e_steps, full)
        e_ev.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(s_ev.elapsed_time(e_ev) / e2e_steps, world, dev)

    e2e_max = e2e_time(False)
    e2e_val = whole_job_tflops(flops, world, e2e_max)
    e2e_full_max = e2e_time(True)
    # the training step through the public API without the pipelining (one
    # step after another on one stream), for reference
    def serial_step():
        b_in[0].copy_(b_host, non_blocking=True)
        dc_in[0].copy_(dc_host, non_blocking=True)
        bb = b_in[0].detach().requires_grad_(True)
        w = w_dev.detach().requires_grad_(True)
        c = routed_spmm(adj, bb, w)
        loss = (c * dc_in[0]).sum()
        loss.backward()
        m_host[0].copy_(torch.stack([loss.detach(), bb.grad.float().square().sum(),
                                     w.grad.square().sum()]), non_blocking=True)
    serial_ms = float(np.mean(timed(serial_step, min(e2e_steps, 10), 2)))

    peak, peak_kind = _peaks()
    if fwd_block:
        res_bytes = res_gbs = None
    else:
        res_nnz = int(pf.info["residual_nnz"])
        res_bytes = algorithmic_bytes(res_nnz, g.n_rows, g.n_cols, k, 4)
        res_gbs = res_bytes / (res_ms * 1e-3) / 1e9
    fwd_bytes = algorithmic_bytes(g.nnz, g.n_rows, g.n_cols, k, 4)
    sbytes = step_bytes(g.nnz, g.n_rows, g.n_cols, k)
    cpu = None
    cpu_torch = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_torch = torch_sparse_cpu_forward(g, b)
        cs = CpuStep(g, gt, b, dc)
        sec, reps = cs.time(budget_s=12.0)
        cpu = {"value": flops / sec / 1e12, "unit": UNIT, "cores": cs.threads, "kind": "port",
               "sample": f"full workload, the whole step (forward, adjoint, SDDMM), "
                         f"{reps} steps in {sec * reps:.1f} s"}
    clocks = clk.summary()
    batched = None
    if rank == 0 and not args.no_batched:
        batched = batched_comparison(dev, flush)
    router = router_comparison(g) if rank == 0 else None

    def launches(p):
        info = p.info
        if info["engine"] == trspmm.TR_ENGINE_BLOCK:
            return 1
        tiles = info["tc_tiles"] + info["sptc_tiles"] + info["promoted_tiles"] > 0
        return (1 if (info["residual_nnz"] > 0 or not tiles) else 0) + (1 if tiles else 0)

    fused_bwd = (pa.info["engine"] == trspmm.TR_ENGINE_WINDOW
                 and pa.info["tc_tiles"] + pa.info["sptc_tiles"] + pa.info["promoted_tiles"] == 0
                 and pa.info["residual_nnz"] == g.nnz and k <= 256)
    # the block engine's tensor-core backward: dB and dval in one launch
    block_bwd = pa.info["engine"] == trspmm.TR_ENGINE_BLOCK and k in (64, 128)
    bwd_launches = 1 if (fused_bwd or block_bwd) else launches(pa) + 1
    # the dominant kernel of the step: the longer of the backward's one fused
    # launch and the forward's (block kernel or CUDA-core residual pass)
    fwd_kernel_ms = fwd_ms if fwd_block else res_ms
    if fused_bwd and adj_sddmm_ms >= fwd_kernel_ms:
        dom_kernel = "seg_adjoint_sddmm_kernel (fused backward: dB = A^T dC, dval = SDDMM)"
        abytes = adjoint_sddmm_bytes(g.nnz, g.n_rows, g.n_cols, k, entry_ids=adj.edge_id is None)
        achieved = abytes / (adj_sddmm_ms * 1e-3) / 1e9
        traffic = _profile_traffic("seg_adjoint_sddmm_large_routed.txt")
    elif block_bwd and adj_sddmm_ms >= fwd_kernel_ms:
        dom_kernel = "block_bwd_kernel (tensor-core backward: dB = A^T dC, dval = SDDMM)"
        abytes = block_bwd_bytes(g.nnz, int(pa.info["chunks"]), g.n_rows, g.n_cols, k,
                                 entry_ids=adj.edge_id is None)
        achieved = abytes / (adj_sddmm_ms * 1e-3) / 1e9
        traffic = _profile_traffic("block_bwd_large_routed.txt")
    elif fwd_block:
        dom_kernel = "block_mma_kernel (forward on the tensor cores, 128-row blocks)"
        abytes, achieved = fwd_bytes, fwd_bytes / (fwd_ms * 1e-3) / 1e9
        traffic = _profile_traffic("block_mma_forward_large_routed.txt")
    else:
        dom_kernel = "seg_block_kernel (forward residual pass)"
        abytes, achieved = res_bytes, res_gbs
        traffic = _profile_traffic("seg_residual_pass_large_routed.txt")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": warm, "ms_per_step": ms_max,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16",
            "data": "synthetic",
            "config": {"workload": args.workload, "n_nodes": g.n_rows, "nnz": g.nnz, "k": k,
                       "step": "forward + adjoint + SDDMM", "out": "f32",
                       "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"replicas{world}", "plan_options": opts,
                       "adjoint_plan_options": adj_opts,
                       "edge_order": ("adjoint plan entry order (A^T CSR)" if adj.edge_id is not None
                                      else "A CSR order")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": peak_kind, "algorithmic_bytes": abytes,
                         "kernel": dom_kernel},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_val, "unit": UNIT,
                    "h2d_bytes_per_step": int(b.nbytes + dc.nbytes),
                    "d2h_bytes_per_step": 12,
                    "ms_per_step": e2e_max,
                    "step": "routed_spmm autograd training step: upload B and the upstream "
                            "gradient G, C = A(w) B, loss <C, G>, backward; result read back: "
                            "the loss and |dB|^2, |dw|^2 (3 FP32)",
                    "pipelined": "step i+1's upload and step i's download overlap step i's "
                                 "compute (two copy streams, two slots)",
                    "serial_ms_per_step": serial_ms},
            "gpu_launches": args.steps * (launches(pf) + bwd_launches),
            "clocks": clocks,
            "extra": {"forward_ms": fwd_ms, "adjoint_ms": adj_ms, "sddmm_ms": sddmm_ms,
                      "adjoint_sddmm_fused_ms": adj_sddmm_ms,
                      "cpu_torch_sparse_forward": cpu_torch,
                      "forward_residual_pass_ms": res_ms,
                      "forward_residual_roofline": None if fwd_block else {
                          "achieved_gbs": res_gbs, "frac": res_gbs / peak,
                          "algorithmic_bytes": res_bytes,
                          "traffic": _profile_traffic("seg_residual_pass_large_routed.txt")},
                      "forward_gathers": None if not fwd_block else {
                          "distinct_block_columns_per_entry": pf.info["slots"] / g.nnz,
                          "l2_to_sm_gather_bytes_per_pass": pf.info["slots"] * k * 2,
                          "window_engine_gather_bytes_per_pass": g.nnz * k * 2},
                      "forward_roofline": {
                          "achieved_gbs": fwd_bytes / (fwd_ms * 1e-3) / 1e9,
                          "frac": fwd_bytes / (fwd_ms * 1e-3) / 1e9 / peak,
                          "algorithmic_bytes": fwd_bytes,
                          "traffic": _profile_traffic("block_mma_forward_large_routed.txt")
                          if fwd_block else None},
                      "plain_csr_step_ms": plain_ms, "plain_csr_forward_ms": plain_fwd_ms,
                      "plain_fused_backward_ms": plain_bwd_ms,
                      "block_tensor_core_backward_ms": block_bwd_ms,
                      "fused_backward_deterministic_ms": det_bwd_ms,
                      "fp32_features_forward": fp32_route,
                      "routed_vs_plain_step": plain_ms / ms,
                      "routed_vs_plain_forward": plain_fwd_ms / fwd_ms,
                      "routed_vs_plain_backward_fused": plain_bwd_ms / adj_sddmm_ms,
                      "routed_vs_plain_step_equal_fusion":
                          (plain_fwd_ms + plain_bwd_ms) / (fwd_ms + adj_sddmm_ms),
                      "max_rel_diff_vs_plain": err,
                      "step_algorithmic_bytes": sbytes,
                      "step_hbm_gbs": sbytes / (ms * 1e-3) / 1e9,
                      "step_hbm_frac": sbytes / (ms * 1e-3) / 1e9 / peak,
                      "plan_build_s": plan_s, "tune_s": tune_s, "router_s": router,
                      "autotune": {
                          "sample": tune_report.get("sample"),
                          "on_sample": [{"options": r["options"], "ms": r["ms"]}
                                        for r in tune_report.get("results", [])],
                          "full_size": [{"options": r["options"], "ms": r["ms"]}
                                        for r in tune_report.get("full", [])]},
                      "autotune_backward": {
                          "sample": bwd_report.get("sample"),
                          "on_sample": [{"options": r["options"], "ms": r["ms"]}
                                        for r in bwd_report.get("results", [])],
                          "full_size": [{"options": r["options"], "ms": r["ms"]}
                                        for r in bwd_report.get("full", [])]},
                      "batched_512": batched,
                      "plan_forward": pf.info, "plan_adjoint": pa.info,
                      "e2e_full_outputs": {
                          "value": whole_job_tflops(flops, world, e2e_full_max), "unit": UNIT,
                          "ms_per_step": e2e_full_max,
                          "d2h_bytes_per_step": int(g.n_rows * k * 4 + g.n_cols * k * 2 + g.nnz * 4),
                          "step": "the same step downloading all of C (FP32), dB (FP16) and dw "
                                  "(FP32) every step"}},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
