"""As-rigid-as-possible regulariser of the embedded graph: drop-in for the
``EmbeddedGraphArapGpu`` op and its gradient op.

Mirrors CustomTensorFlowCPPOperators/src/CustomGPUOperators/
EmbeddedGraphARAPOperator/EmbeddedGraphArapGPUOp.cpp:5-16 and
EmbeddedGraphArapGPUOpGrad.cpp:5-15: inputs nodes_translation and
nodes_rotation (Euler, rad) [B,M,3]; outputs nodes_arap_loss
[B,M,max_connections,3], d_connection_weights [B,M,max_connections] and
d_rotation [B,M,3]; gradients to the translations and rotations only.  The
op reads the base mesh, the node neighbours and the rigidity weights from the
character / graph files; here they are passed as arrays (what those loaders
produce; ``synthetic.node_graph`` builds them for a synthetic graph).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .renderer import _f32, _stream


class ArapEngine:
    """Owns one ``hc_arap`` handle."""

    def __init__(self, base_vertices, node_vertex, n2n_offsets, n2n_sizes, n2n_indices, rigidity,
                 max_connections: int):
        arr = lambda a, dt: np.ascontiguousarray(np.asarray(a, dt))  # noqa: E731
        self._keep = [arr(base_vertices, np.float32), arr(node_vertex, np.int32), arr(n2n_offsets, np.int32),
                      arr(n2n_sizes, np.int32), arr(n2n_indices, np.int32), arr(rigidity, np.float32)]
        k = self._keep
        self.N, self.M, self.maxc = k[0].shape[0], k[1].shape[0], int(max_connections)
        h = C.c_void_p()
        P = _lib.ptr
        _lib.call("hc_arap_create", C.byref(h), self.N, P(k[0]), self.M, P(k[1]), P(k[2]), P(k[3]), P(k[4]), P(k[5]),
                  self.maxc)
        self._h = h

    @classmethod
    def from_graph_file(cls, graph) -> "ArapEngine":
        """From a ``loaders.GraphFile`` (graph-mesh neighbours, segmentation rigidity)."""
        return cls(graph.eg.base_vertices, graph.eg.node_vertex, graph.n2n_offsets, graph.n2n_sizes,
                   graph.n2n_indices, graph.rigidity, graph.max_connections)

    @classmethod
    def from_graph(cls, base_vertices, node_vertex, g):
        """From a ``synthetic.NodeGraph`` (or any object with its fields)."""
        return cls(base_vertices, node_vertex, g.n2n_offsets, g.n2n_sizes, g.n2n_indices, g.rigidity,
                   g.max_connections)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib.lib().hc_arap_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def forward(self, nodes_translation, nodes_rotation):
        T, A = _f32(nodes_translation, "nodes_translation"), _f32(nodes_rotation, "nodes_rotation")
        if T.shape[1:] != (self.M, 3) or A.shape != T.shape:
            raise ValueError(f"nodes_translation / nodes_rotation must be [B,{self.M},3]")
        B, dev = T.shape[0], T.device
        loss = torch.empty((B, self.M, self.maxc, 3), device=dev)
        w = torch.empty((B, self.M, self.maxc), device=dev)
        rot = torch.empty((B, self.M, 3), device=dev)
        P = _lib.ptr
        _lib.call("hc_arap_forward", self._h, _stream(), B, P(T), P(A), P(loss), P(w), P(rot))
        return loss, w, rot

    def backward(self, nodes_arap_loss_grad, d_rotation):
        g, A = _f32(nodes_arap_loss_grad, "nodes_arap_loss_grad"), _f32(d_rotation, "d_rotation")
        B, dev = A.shape[0], A.device
        if g.shape != (B, self.M, self.maxc, 3):
            raise ValueError(f"nodes_arap_loss_grad must be [B,{self.M},{self.maxc},3]")
        gT = torch.empty((B, self.M, 3), device=dev)
        gA = torch.empty((B, self.M, 3), device=dev)
        P = _lib.ptr
        _lib.call("hc_arap_backward", self._h, _stream(), B, P(g), P(A), P(gT), P(gA))
        return gT, gA


class _ArapFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eng: ArapEngine, T, A):
        loss, w, rot = eng.forward(T, A)
        ctx.eng = eng
        ctx.save_for_backward(rot)
        ctx.mark_non_differentiable(w, rot)
        return loss, w, rot

    @staticmethod
    def backward(ctx, gl, gw, gr):
        (rot,) = ctx.saved_tensors
        if gl is None:
            return None, None, None
        gT, gA = ctx.eng.backward(gl, rot)
        return None, gT, gA


def embedded_graph_arap(engine: ArapEngine, nodes_translation, nodes_rotation):
    """(nodes_arap_loss, d_connection_weights, d_rotation), differentiable in
    the translations and rotations through ``hc_arap_backward``."""
    return _ArapFn.apply(engine, nodes_translation, nodes_rotation)
