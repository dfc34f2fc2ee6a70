"""Differentiable PageRank for PyTorch (no reference counterpart).

``pagerank(graph, weights, teleport=None, ...)`` returns the PageRank scores
of a weighted graph (the forward of nkg_pagerank_run_ex, normalized=False) as
a float64 tensor on the graph's device, differentiable with respect to the
arc weights and the teleport vector. The backward pass is the adjoint solve
of nkg_pagerank_adjoint: one transposed fixed-point solve per backward call,
whatever the number of arcs, instead of one forward solve per weight.

Weights are in the order of the ``in_col`` array the graph was created from;
the teleport vector has ``upperNodeIdBound()`` entries. All tensors must be
float64 CUDA tensors on the graph's device; nothing crosses PCIe but the
iteration status.
"""
from __future__ import annotations

import torch

from . import _capi

_PRECISIONS = {"fp64": _capi.NKG_PREC_FP64, "fp32_refine": _capi.NKG_PREC_FP32_REFINE,
               "fp32": _capi.NKG_PREC_FP32}


class DifferentiableGraph:
    """A weighted graph resident on one GPU whose arc weights are replaced on
    every forward call (nkg_graph_set_weights keeps the layout)."""

    def __init__(self, csr, device: int = 0):
        if csr.in_w is None:
            raise ValueError("the differentiable form needs a weighted graph (in_w)")
        self.graph = _capi.DeviceGraph(csr, device=device)
        self.device = torch.device("cuda", device)
        self.z = int(csr.z)
        self.arcs = int(csr.in_col.shape[0])
        self.loaded_by = None  # the forward call whose weights the graph holds

    def load_weights(self, w: torch.Tensor, token) -> None:
        """Copy `w` into the graph for the forward call `token`. Every forward
        copies (a tensor can change in place without a new version, e.g.
        through .data); a backward copies only if another forward ran since
        its own (autograd itself rejects in-place changes of saved weights)."""
        if token is not None and self.loaded_by is token:
            return
        _check_tensor(w, self.arcs, self.device, "weights")
        torch.cuda.current_stream(self.device).synchronize()
        self.graph.set_weights_device(w.data_ptr())
        self.loaded_by = token


def _check_tensor(t, size, device, name):
    if t.dtype != torch.float64 or t.device != device or t.dim() != 1 or t.shape[0] != size:
        raise ValueError(f"{name} must be a float64 tensor of {size} entries on {device}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def _params(damp, tol, distribute, precision, max_iterations):
    # L1 stopping test, normalized = False (the form the adjoint covers)
    return _capi.PRParams(float(damp), float(tol), 0, 0, int(bool(distribute)), int(precision),
                          int(max_iterations))


class _PageRankFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, weights, teleport, graph, fwd, bwd):
        token = object()
        graph.load_weights(weights, None)
        graph.loaded_by = token
        ctx.token = token
        if teleport is not None:
            _check_tensor(teleport, graph.z, graph.device, "teleport")
        out = torch.empty(graph.z, dtype=torch.float64, device=graph.device)
        torch.cuda.current_stream(graph.device).synchronize()
        tp = teleport.data_ptr() if teleport is not None else 0
        graph.graph.run_ex(fwd, tp, out.data_ptr(), True)
        ctx.graph = graph
        ctx.bwd = bwd
        ctx.has_teleport = teleport is not None
        ctx.save_for_backward(weights, teleport if teleport is not None else out.new_empty(0),
                              out)
        return out

    @staticmethod
    def backward(ctx, grad_out):
        weights, teleport, scores = ctx.saved_tensors
        graph = ctx.graph
        graph.load_weights(weights, ctx.token)
        g = grad_out.contiguous().to(torch.float64)
        want_w = ctx.needs_input_grad[0]
        want_t = ctx.needs_input_grad[1]
        gw = torch.empty(graph.arcs, dtype=torch.float64, device=graph.device) if want_w else None
        gt = torch.empty(graph.z, dtype=torch.float64, device=graph.device) if want_t else None
        torch.cuda.current_stream(graph.device).synchronize()
        graph.graph.adjoint_device(ctx.bwd, scores.data_ptr(), g.data_ptr(),
                                   gw.data_ptr() if gw is not None else 0,
                                   gt.data_ptr() if gt is not None else 0,
                                   teleport.data_ptr() if ctx.has_teleport else 0)
        return gw, gt, None, None, None


def pagerank(graph: DifferentiableGraph, weights: torch.Tensor, teleport: torch.Tensor = None,
             damp: float = 0.85, tol: float = 1e-10, distribute_sinks: bool = True,
             precision: str = "fp32_refine", backward_precision: str = None,
             backward_tol: float = None, max_iterations: int = _capi.UINT64_MAX) -> torch.Tensor:
    """PageRank scores (sum 1) of `graph` with arc weights `weights` and an
    optional teleport distribution; differentiable in both. `precision` picks
    the forward arithmetic ("fp64", "fp32_refine", "fp32"); the backward uses
    `backward_precision` (default: the same) to relative tolerance
    `backward_tol` (default: tol)."""
    fwd = _params(damp, tol, distribute_sinks, _PRECISIONS[precision], max_iterations)
    bwd = _params(damp, tol if backward_tol is None else backward_tol, distribute_sinks,
                  _PRECISIONS[backward_precision or precision], max_iterations)
    return _PageRankFn.apply(weights, teleport, graph, fwd, bwd)
