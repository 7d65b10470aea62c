"""Many small graphs in one launch.

A batch of independent graphs of uneven sizes (node offsets per graph) is
one block-diagonal sparse matrix: one routed plan (and one adjoint plan)
covers every graph, so the forward and the fused backward of the whole batch
are one residual pass, at most one tile pass and one fused adjoint/SDDMM
pass — and the whole step can be captured once in a CUDA graph and replayed
as a single launch.  ``PerGraphLoop`` is the comparison a per-graph library
call gives: one plan pair per graph and one launch sequence per graph.

The reference has no batching (one graph per operator call).
"""
from __future__ import annotations

import numpy as np
import torch

from .autograd import RoutedAdjacency


class BatchedStep:
    """Forward C = A B and backward (dB, dval) of a block-diagonal batch on
    static device buffers, optionally captured in a CUDA graph."""

    def __init__(self, g, k, device="cuda", **plan_opts):
        self.g = g
        self.k = int(k)
        self.dev = torch.device(device)
        self.adj = RoutedAdjacency(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                                   device=self.dev, **plan_opts)
        self.b = torch.empty((g.n_cols, self.k), dtype=torch.float16, device=self.dev)
        self.dc = torch.empty((g.n_rows, self.k), dtype=torch.float16, device=self.dev)
        self.c = torch.empty((g.n_rows, self.k), dtype=torch.float32, device=self.dev)
        self.db = torch.empty((g.n_cols, self.k), dtype=torch.float32, device=self.dev)
        self.dval = torch.empty(g.nnz, dtype=torch.float32, device=self.dev)
        self.graph = None

    def run(self):
        a = self.adj
        a.fwd.spmm(self.b, out=self.c)
        a.adj.adjoint_sddmm(a.indptr, a.indices, self.dc, self.b, db=self.db, dval=self.dval)

    def capture(self, warmup=2):
        """Record run() into a CUDA graph (after warm-up launches on a side
        stream, as capture requires)."""
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self.run()
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.run()
        return self

    def replay(self):
        if self.graph is None:
            self.run()
        else:
            self.graph.replay()


class PerGraphLoop:
    """The same step as a loop over the graphs, one plan pair each."""

    def __init__(self, g, k, device="cuda", **plan_opts):
        if g.offsets is None:
            raise ValueError("the batch needs per-graph node offsets")
        self.g = g
        self.k = int(k)
        self.dev = torch.device(device)
        off = np.asarray(g.offsets, dtype=np.int64)
        self.parts = []
        for i in range(len(off) - 1):
            r0, r1 = int(off[i]), int(off[i + 1])
            e0, e1 = int(g.indptr[r0]), int(g.indptr[r1])
            ip = (g.indptr[r0:r1 + 1] - e0).astype(np.int32)
            ix = (g.indices[e0:e1] - r0).astype(np.int32)
            vv = g.values[e0:e1]
            adj = RoutedAdjacency(ip, ix, vv, r1 - r0, r1 - r0, device=self.dev, **plan_opts)
            self.parts.append((r0, r1, e0, e1, adj))
        self.b = torch.empty((g.n_cols, self.k), dtype=torch.float16, device=self.dev)
        self.dc = torch.empty((g.n_rows, self.k), dtype=torch.float16, device=self.dev)
        self.c = torch.empty((g.n_rows, self.k), dtype=torch.float32, device=self.dev)
        self.db = torch.empty((g.n_cols, self.k), dtype=torch.float32, device=self.dev)
        self.dval = torch.empty(g.nnz, dtype=torch.float32, device=self.dev)

        self.graph = None

    def run(self):
        for r0, r1, e0, e1, a in self.parts:
            a.fwd.spmm(self.b[r0:r1], out=self.c[r0:r1])
            a.adj.adjoint_sddmm(a.indptr, a.indices, self.dc[r0:r1], self.b[r0:r1],
                                db=self.db[r0:r1], dval=self.dval[e0:e1])

    def capture(self, warmup=2):
        """The loop's launches recorded in one CUDA graph (removes the host
        cost of issuing them; the device still runs one kernel sequence per
        graph)."""
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self.run()
        torch.cuda.current_stream(self.dev).wait_stream(s)
        torch.cuda.synchronize(self.dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.run()
        return self

    def replay(self):
        if self.graph is None:
            self.run()
        else:
            self.graph.replay()
