"""Differentiable personalized PageRank (torch.autograd.Function).

    s = PageRankFunction.apply(teleport, edge_w, graph_ctx)

returns the fixed point s = (1-d) t + d P^T s, P[v,u] = w(v->u) / S_v, of the
GPU engine, and its backward pass runs the engine's adjoint:
    lambda = grad_s + d P lambda            (gather over out-neighbours)
    dL/dt         = (1-d) lambda
    dL/dw(v->u)   = d s[v] / S_v (lambda[u] - (P lambda)[v])
with edge_w aligned with the graph's out-CSR.  All tensors live on the
engine's CUDA device (float32).  The graph is uploaded once; new edge
weights (a training step) go to the engine from device memory
(pr_gpu_set_edge_weights_device), with no host round trip.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from .graph import Graph
from .pagerank import K_DAMP, PageRankEngine


@dataclass
class PageRankContext:
    """Engine + graph + solver settings shared by forward and backward."""
    graph: Graph
    device: int = 0
    max_iters: int = 100
    epsilon: float = 1e-6
    damping: float = float(K_DAMP)
    adjoint_max_iters: int = 300
    adjoint_epsilon: float = 1e-6
    engine: PageRankEngine = field(init=False)
    _weights_key: Optional[tuple] = field(default=None, init=False)
    last_sweeps: int = field(default=0, init=False)
    last_adjoint_sweeps: int = field(default=0, init=False)
    uploads: int = field(default=0, init=False)          # full graph uploads
    weight_updates: int = field(default=0, init=False)   # device weight updates

    def __post_init__(self):
        self.engine = PageRankEngine(self.device)

    def ensure_weights(self, edge_w: Optional[torch.Tensor]):
        """Puts edge_w (or unit weights for None) in the engine: a full
        upload the first time and when switching between weighted and
        unweighted, else a device-to-device weight update."""
        key = None if edge_w is None else (edge_w.data_ptr(), edge_w._version, edge_w.numel())
        if self._weights_key is not None and key == self._weights_key[0]:
            return
        was_weighted = self._weights_key is not None and self._weights_key[0] is not None
        if edge_w is not None and was_weighted:
            if edge_w.numel() != self.engine.m:
                raise ValueError("edge_w must have one entry per directed edge")
            w = _cuda_f32(edge_w, self.device)
            torch.cuda.current_stream(w.device).synchronize()
            self.engine.set_edge_weights_device(w.data_ptr())
            self.weight_updates += 1
        else:
            w = None if edge_w is None else edge_w.detach().float().cpu().numpy()
            self.engine.upload(self.graph, edge_w=w)
            self.uploads += 1
        self._weights_key = (key,)


def _cuda_f32(x: torch.Tensor, dev: int) -> torch.Tensor:
    return x.detach().to(device=f"cuda:{dev}", dtype=torch.float32).contiguous()


class PageRankFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, teleport: torch.Tensor, edge_w: Optional[torch.Tensor],
                pctx: PageRankContext):
        pctx.ensure_weights(edge_w)
        eng = pctx.engine
        t = _cuda_f32(teleport, pctx.device)
        if t.numel() != eng.n:
            raise ValueError("teleport must have one entry per vertex")
        out = torch.empty(eng.n, device=t.device, dtype=torch.float32)
        torch.cuda.current_stream(t.device).synchronize()
        sweeps, _ = eng.run_device(pctx.max_iters, pctx.epsilon, pctx.damping, 1,
                                   t.data_ptr(), out.data_ptr())
        pctx.last_sweeps = int(sweeps[0])
        ctx.pctx = pctx
        ctx.has_w = edge_w is not None
        ctx.save_for_backward(out)
        return out

    @staticmethod
    def backward(ctx, grad_s: torch.Tensor):
        (s,) = ctx.saved_tensors
        pctx: PageRankContext = ctx.pctx
        eng = pctx.engine
        gs = _cuda_f32(grad_s, pctx.device)
        grad_t = torch.empty(eng.n, device=gs.device, dtype=torch.float32)
        want_w = ctx.has_w and ctx.needs_input_grad[1]
        grad_w = torch.empty(eng.m, device=gs.device, dtype=torch.float32) if want_w else None
        torch.cuda.current_stream(gs.device).synchronize()
        pctx.last_adjoint_sweeps = eng.adjoint_device(
            pctx.adjoint_max_iters, pctx.adjoint_epsilon, pctx.damping, gs.data_ptr(),
            s.data_ptr(), grad_t.data_ptr(), None if grad_w is None else grad_w.data_ptr())
        return grad_t, grad_w, None


def personalized_pagerank(teleport: torch.Tensor, edge_w: Optional[torch.Tensor],
                          pctx: PageRankContext) -> torch.Tensor:
    return PageRankFunction.apply(teleport, edge_w, pctx)


__all__ = ["PageRankContext", "PageRankFunction", "personalized_pagerank"]
