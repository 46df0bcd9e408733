"""Embedded-graph deformation: drop-in for ``EmbeddedGraphGpu``.

Mirrors Projects/CustomTFOperators/EmbeddedGraphGpu.py:21-94 and the op
(CustomTensorFlowCPPOperators/src/CustomGPUOperators/EmbeddedGraphOperator/
EmbeddedGraphGPUOp.cpp:6-25, EmbeddedGraphGPUOpGrad.cpp:5-21): same inputs
(node delta / skinned translations and Euler rotations, per-vertex
displacements), same outputs (deformed vertices, normals, markers, graph
nodes) and the same gradient rule (skinned gradients are zero unless the
full mode is requested).  The reference reads the base mesh and graph from
character / graph files; here they are passed as arrays (``EGData``), which
is what those loaders produce.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np
import torch

from . import _lib
from .renderer import _f32, _stream


@dataclasses.dataclass
class EGData:
    """Arrays of a skinned character's embedded graph (Skeletool/Mesh/EmbeddedGraph.cpp:379-548)."""
    base_vertices: np.ndarray           # [N,3] float32 (mm)
    faces: np.ndarray                   # [F,3] int32
    node_vertex: np.ndarray             # [M] int32
    v2n_offsets: np.ndarray
    v2n_sizes: np.ndarray
    v2n_indices: np.ndarray
    v2n_weights: np.ndarray
    n2v_offsets: np.ndarray
    n2v_sizes: np.ndarray
    n2v_indices: np.ndarray
    n2v_weights: np.ndarray
    markers: np.ndarray | None = None   # [Mk,3]
    marker_node: np.ndarray | None = None  # [Mk]

    @classmethod
    def from_synthetic(cls, verts, faces, graph, markers=None, marker_node=None):
        return cls(np.asarray(verts, np.float32), np.asarray(faces, np.int32), graph.node_vertex, graph.v2n_offsets,
                   graph.v2n_sizes, graph.v2n_indices, graph.v2n_weights, graph.n2v_offsets, graph.n2v_sizes,
                   graph.n2v_indices, graph.n2v_weights, markers, marker_node)


class EmbeddedGraphEngine:
    """Owns one ``hc_eg`` handle."""

    def __init__(self, data: EGData, full_skinned_gradient: bool = False):
        self.data = data
        arr = lambda a, dt: np.ascontiguousarray(np.asarray(a, dt))  # noqa: E731
        self._keep = [arr(data.base_vertices, np.float32), arr(data.faces, np.int32), arr(data.node_vertex, np.int32),
                      arr(data.v2n_offsets, np.int32), arr(data.v2n_sizes, np.int32), arr(data.v2n_indices, np.int32),
                      arr(data.v2n_weights, np.float32), arr(data.n2v_offsets, np.int32),
                      arr(data.n2v_sizes, np.int32), arr(data.n2v_indices, np.int32),
                      arr(data.n2v_weights, np.float32)]
        mk = None if data.markers is None else arr(data.markers, np.float32)
        mn = None if data.marker_node is None else arr(data.marker_node, np.int32)
        self._keep += [mk, mn]
        k = self._keep
        self.N = k[0].shape[0]
        self.F = k[1].size // 3
        self.M = k[2].shape[0]
        self.Mk = 0 if mk is None else mk.shape[0]
        h = C.c_void_p()
        P = _lib.ptr
        _lib.call("hc_eg_create", C.byref(h), self.N, P(k[0]), P(k[1]), self.F, self.M, P(k[2]), P(k[3]), P(k[4]),
                  P(k[5]), P(k[6]), P(k[7]), P(k[8]), P(k[9]), P(k[10]), self.Mk, P(mk), P(mn))
        self._h = h
        self.full = bool(full_skinned_gradient)
        _lib.call("hc_eg_set_full_skinned_gradient", h, int(self.full))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib.lib().hc_eg_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def reserve(self, batch: int):
        _lib.call("hc_eg_reserve", self._h, int(batch))

    def forward(self, dT, dA, sT, sA, disp, out: dict | None = None):
        dT, dA, sT, sA, disp = (_f32(t, n) for t, n in ((dT, "nodes_delta_translation"), (dA, "nodes_delta_rotation"),
                                                        (sT, "nodes_skinned_translation"),
                                                        (sA, "nodes_skinned_rotation"),
                                                        (disp, "vertex_displacements")))
        B = dT.shape[0]
        dev = dT.device
        o = out or {}
        e = lambda k, shape: o[k] if o.get(k) is not None else torch.empty(shape, device=dev)  # noqa: E731
        v = e("vertices", (B, self.N, 3))
        n = e("normals", (B, self.N, 3))
        m = e("markers", (B, self.Mk, 3))
        g = e("graph", (B, self.M, 3))
        da = e("d_delta_rotation", (B, self.M, 3))
        sa = e("d_skinned_rotation", (B, self.M, 3))
        P = _lib.ptr
        _lib.call("hc_eg_forward", self._h, _stream(), B, P(dT), P(dA), P(sT), P(sA), P(disp), P(v), P(n),
                  P(m) if self.Mk else None, P(g), P(da), P(sa))
        return v, n, m, g, da, sa

    def backward(self, gv, gm, da, sa, dT=None, disp=None):
        gv = _f32(gv, "deformed_vertices_grad")
        B = gv.shape[0]
        dev = gv.device
        gm = _f32(gm, "deformed_markers_grad") if (gm is not None and self.Mk) else None
        da, sa = _f32(da, "d_delta_a"), _f32(sa, "d_skinned_a")
        out = [torch.empty((B, self.M, 3), device=dev) for _ in range(4)]
        gd = torch.empty((B, self.N, 3), device=dev)
        P = _lib.ptr
        _lib.call("hc_eg_backward", self._h, _stream(), B, P(gv), P(gm), P(da), P(sa), *(P(t) for t in out), P(gd),
                  P(_f32(dT, "dT")) if self.full else None, P(_f32(disp, "disp")) if self.full else None)
        return out[0], out[1], out[2], out[3], gd


class _EGFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eng: EmbeddedGraphEngine, dT, dA, sT, sA, disp):
        v, n, m, g, da, sa = eng.forward(dT, dA, sT, sA, disp)
        ctx.eng = eng
        ctx.save_for_backward(da, sa, dT, disp)
        ctx.mark_non_differentiable(da, sa)
        return v, n, m, g, da, sa

    @staticmethod
    def backward(ctx, gv, gn, gm, gg, gda, gsa):
        da, sa, dT, disp = ctx.saved_tensors
        eng: EmbeddedGraphEngine = ctx.eng
        if gv is None:
            gv = torch.zeros((da.shape[0], eng.N, 3), device=da.device)
        # the reference gradient ignores the normal and graph-node outputs
        # (EmbeddedGraphGpu.py:82-94)
        tg, rg, stg, srg, dg = eng.backward(gv, gm, da, sa, dT, disp)
        return None, tg, rg, stg, srg, dg


class EmbeddedGraphGpu:
    """Reference-shaped wrapper (Projects/CustomTFOperators/EmbeddedGraphGpu.py:21-76).

    Without ``graph_data`` or ``engine`` the graph is built from
    ``characterFilePath`` and ``graphFilePath`` as the reference op does
    (EmbeddedGraphGPUOp.cpp:22-60), with ``loaders.load_character`` and
    ``loaders.load_graph``."""

    def __init__(self, characterFilePath="", graphFilePath="", numberOfBatches=0, deltaT=None, deltaR=None,
                 skinnedT=None, skinnedR=None, displacements=None, refinement=None, nodeName="",
                 graph_data: EGData | None = None, engine: EmbeddedGraphEngine | None = None,
                 full_skinned_gradient: bool = False):
        if engine is None:
            if graph_data is None and characterFilePath and graphFilePath:
                from . import loaders
                graph_data = loaders.load_graph(loaders.load_character(characterFilePath), graphFilePath,
                                                bool(refinement)).eg
            if graph_data is None:
                raise ValueError("Invalid argument during the construction of the embedded graph operator! "
                                 "(pass characterFilePath and graphFilePath, or graph_data=)")
            engine = EmbeddedGraphEngine(graph_data, full_skinned_gradient)
        if any(t is None for t in (deltaT, deltaR, skinnedT, skinnedR, displacements)):
            raise ValueError("Invalid argument during the construction of the embedded graph operator!")
        self.numberOfBatches = numberOfBatches
        self.nodeName = nodeName
        self.engine = engine
        self.embeddedGraphGpuOperator = _EGFn.apply(engine, deltaT, deltaR, skinnedT, skinnedR, displacements)

    def getNode(self):
        o = self.embeddedGraphGpuOperator
        return [o[0], o[1], o[2], o[3]]
