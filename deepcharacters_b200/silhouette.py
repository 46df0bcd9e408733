"""Camera projection, projected-mesh boundary and the multi-view silhouette
distance-transform loss.

Drop-ins for ``CameraProjectionGpu`` (Projects/CustomTFOperators/
CameraProjectionGPU.py:20-71; op CameraProjectionGPUOp.cpp:5-12),
``ProjectedMeshBoundaryGpu`` (ProjectedMeshBoundaryGPUOp.cpp:5-18) and
``MultiViewSilhouetteLossGpu`` (MultiViewSilhouetteLossGPUOp.cpp:5-14) with
their registered gradients.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .renderer import _f32, _stream


def camera_projection_forward(points, vectors, extrinsics, intrinsics, is_point: bool):
    p = _f32(points, "points_global_space")
    v = _f32(vectors, "vectors_global_space") if vectors is not None else None
    ex, it = _f32(extrinsics, "extrinsics"), _f32(intrinsics, "intrinsics")
    B, N = p.shape[0], p.shape[1]
    Cn = ex.reshape(B, -1).shape[1] // 12
    out = torch.empty((B, Cn, N, 2), device=p.device)
    P = _lib.ptr
    _lib.call("hc_camera_projection_forward", _stream(), B, Cn, N, P(p), P(v), P(ex), P(it), int(is_point), P(out))
    return out


def camera_projection_backward(grad, points, extrinsics, intrinsics, is_point: bool):
    g, p = _f32(grad, "grad"), _f32(points, "points_global_space")
    ex, it = _f32(extrinsics, "extrinsics"), _f32(intrinsics, "intrinsics")
    B, Cn, N = g.shape[0], g.shape[1], g.shape[2]
    out = torch.empty((B, N, 3), device=g.device)
    P = _lib.ptr
    _lib.call("hc_camera_projection_backward", _stream(), B, Cn, N, P(g), P(p), P(ex), P(it), int(is_point), P(out))
    return out


class _ProjFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, points, vectors, extrinsics, intrinsics, is_point):
        ctx.save_for_backward(points, vectors, extrinsics, intrinsics)
        ctx.is_point = bool(is_point)
        return camera_projection_forward(points, vectors, extrinsics, intrinsics, is_point)

    @staticmethod
    def backward(ctx, g):
        points, vectors, extrinsics, intrinsics = ctx.saved_tensors
        gp = camera_projection_backward(g, points, extrinsics, intrinsics, ctx.is_point)
        # normals / cameras get zero gradients (CameraProjectionGPU.py:60-71)
        return (gp, None if vectors is None else torch.zeros_like(vectors), torch.zeros_like(extrinsics),
                torch.zeros_like(intrinsics), None)


class CameraProjectionGpu:
    """Reference-shaped wrapper (Projects/CustomTFOperators/CameraProjectionGPU.py:20-55)."""

    def __init__(self, isPoint=False, pointsGlobalSpace=None, vectorsGlobalSpace=None, extrinsics=None,
                 intrinsics=None, nodeName=""):
        if pointsGlobalSpace is None or extrinsics is None or intrinsics is None:
            raise ValueError("Invalid argument during the construction of the camera projection operator!")
        self.isPoint = isPoint
        self.cameraProjectionGpuOperator = _ProjFn.apply(pointsGlobalSpace, vectorsGlobalSpace, extrinsics,
                                                         intrinsics, bool(isPoint))

    def getNode(self):
        return self.cameraProjectionGpuOperator


def projected_mesh_boundary(points_image_space, face_buffer, width: int, height: int):
    """Boundary flags [B,C,N] (uint8) from image-space points and a renderer face buffer."""
    p = _f32(points_image_space, "points_image_space")
    B, Cn, N = p.shape[0], p.shape[1], p.shape[2]
    out = torch.empty((B, Cn, N), device=p.device, dtype=torch.uint8)
    f = face_buffer.detach().to(torch.int32).contiguous()
    P = _lib.ptr
    _lib.call("hc_projected_mesh_boundary", _stream(), B, Cn, N, int(width), int(height), P(p), P(f), P(out))
    return out


class MeshBoundaryEngine:
    """Owns one ``hc_mesh_boundary`` handle: the mesh faces plus the
    projection / coverage workspaces of ``ProjectedMeshBoundaryGpu``."""

    def __init__(self, faces, n_vertices: int):
        import numpy as np
        f = np.ascontiguousarray(np.asarray(faces, np.int32).reshape(-1, 3))
        self.F, self.N = int(f.shape[0]), int(n_vertices)
        h = C.c_void_p()
        _lib.call("hc_mesh_boundary_create", C.byref(h), f.ctypes.data, self.F, self.N)
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib.lib().hc_mesh_boundary_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def reserve(self, B, Cn, width, height):
        _lib.call("hc_mesh_boundary_reserve", self._h, B, Cn, int(width), int(height))

    def reserve_sized(self, B, Cn, widths, heights):
        w, h = _sizes(widths, heights, Cn)
        _lib.call("hc_mesh_boundary_reserve_sized", self._h, B, Cn, w.ctypes.data, h.ctypes.data)

    def forward_sized(self, points_global_space, extrinsics, intrinsics, widths, heights, points_image_space=None,
                      out=None, face_hint=None):
        """Cameras of different sizes (widths / heights [C]): is_boundary [B,C,N]
        (uint8); ``face_hint`` [B, pixels of a frame] int32 or None."""
        p = _f32(points_global_space, "points_global_space")
        ex, it = _f32(extrinsics, "extrinsics"), _f32(intrinsics, "intrinsics")
        B = p.shape[0]
        Cn = ex.reshape(B, -1).shape[1] // 12
        w, h = _sizes(widths, heights, Cn)
        if out is None:
            out = torch.empty((B, Cn, self.N), device=p.device, dtype=torch.uint8)
        if face_hint is not None and (face_hint.dtype != torch.int32 or not face_hint.is_contiguous()
                                      or face_hint.numel() != B * int((w.astype(np.int64) * h).sum())):
            raise ValueError("face_hint must be a contiguous int32 [B, pixels of a frame] tensor")
        pis = _f32(points_image_space, "points_image_space") if points_image_space is not None else None
        P = _lib.ptr
        _lib.call("hc_mesh_boundary_forward_sized", self._h, _stream(), B, Cn, w.ctypes.data, h.ctypes.data, P(p),
                  P(ex), P(it), P(pis) if pis is not None else None, P(face_hint) if face_hint is not None else None,
                  P(out))
        return out

    def forward(self, points_global_space, extrinsics, intrinsics, width: int, height: int,
                points_image_space=None, out=None, face_hint=None):
        """is_boundary [B,C,N] (uint8).  ``face_hint`` [B,C,H,W] int32 (a renderer
        face buffer of the same views) only saves work: the flags are the same
        for any hint."""
        p = _f32(points_global_space, "points_global_space")
        ex, it = _f32(extrinsics, "extrinsics"), _f32(intrinsics, "intrinsics")
        B = p.shape[0]
        Cn = ex.reshape(B, -1).shape[1] // 12
        if p.shape[1] != self.N:
            raise ValueError(f"points_global_space must be [B,{self.N},3]")
        if out is None:
            out = torch.empty((B, Cn, self.N), device=p.device, dtype=torch.uint8)
        pis = _f32(points_image_space, "points_image_space") if points_image_space is not None else None
        P = _lib.ptr
        if face_hint is None:
            _lib.call("hc_mesh_boundary_forward", self._h, _stream(), B, Cn, int(width), int(height), P(p), P(ex),
                      P(it), P(pis) if pis is not None else None, P(out))
            return out
        if (face_hint.dtype != torch.int32 or not face_hint.is_contiguous()
                or face_hint.numel() != B * Cn * int(width) * int(height)):
            raise ValueError("face_hint must be a contiguous int32 [B,C,H,W] tensor")
        _lib.call("hc_mesh_boundary_forward_hinted", self._h, _stream(), B, Cn, int(width), int(height), P(p), P(ex),
                  P(it), P(pis) if pis is not None else None, P(face_hint), P(out))
        return out


class ProjectedMeshBoundaryGpu:
    """Reference-shaped op (ProjectedMeshBoundaryGPUOp.cpp:5-17): faces stand in
    for ``mesh_file_path_boundary_check``; output is_boundary [B,C,N] (uint8)."""

    def __init__(self, faces, pointsGlobalSpace, extrinsics, intrinsics, numberBatches: int, numberCameras: int,
                 renderU: int, renderV: int, useGapDetection: bool = False, engine: MeshBoundaryEngine | None = None):
        eng = engine or MeshBoundaryEngine(faces, pointsGlobalSpace.shape[1])
        self.isBoundary = eng.forward(pointsGlobalSpace, extrinsics, intrinsics, renderU, renderV)

    def getNode(self):
        return self.isBoundary


class SilhouetteEngine:
    """Owns one ``hc_silhouette`` handle (its boundary-vertex grid workspace)."""

    def __init__(self):
        h = C.c_void_p()
        _lib.call("hc_silhouette_create", C.byref(h))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib.lib().hc_silhouette_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def reserve(self, B, Cn, N, U, V):
        _lib.call("hc_silhouette_reserve", self._h, B, Cn, N, U, V)

    def reserve_sized(self, B, Cn, N, widths, heights):
        w, h = _sizes(widths, heights, Cn)
        _lib.call("hc_silhouette_reserve_sized", self._h, B, Cn, N, w.ctypes.data, h.ctypes.data)

    def forward_sized(self, points, normals, is_boundary, dt, crops, widths, heights):
        """Cameras of different sizes (widths U / heights V [C]): ``dt`` [B, pixels
        of a frame] uint8 (each camera's V_c x U_c image in camera order);
        returns (mv_dt_residual [B,C,N], mv_dt_residual_1 [B, pixels, 2],
        dt_image_gradient [B,C,N,2], closest_vertex_id [B, pixels])."""
        p, n = _f32(points, "points_image_space"), _f32(normals, "normals_image_space")
        isb = is_boundary.detach().to(torch.uint8).contiguous()
        dt = dt.detach().to(torch.uint8).contiguous()
        cr = _f32(crops, "multi_view_crops")
        B, Cn, N = p.shape[0], p.shape[1], p.shape[2]
        w, h = _sizes(widths, heights, Cn)
        pf = int((w.astype(np.int64) * h).sum())
        if dt.numel() != B * pf:
            raise ValueError(f"distance images must hold B x {pf} pixels")
        dev = p.device
        res, res1 = torch.empty((B, Cn, N), device=dev), torch.empty((B, pf, 2), device=dev)
        dtg, cid = torch.empty((B, Cn, N, 2), device=dev), torch.empty((B, pf), device=dev)
        P = _lib.ptr
        _lib.call("hc_silhouette_forward_sized", self._h, _stream(), B, Cn, N, w.ctypes.data, h.ctypes.data, P(p),
                  P(n), P(isb), P(dt), P(cr), P(res), P(res1), P(dtg), P(cid))
        return res, res1, dtg, cid

    def forward(self, points, normals, is_boundary, dt, crops):
        p, n = _f32(points, "points_image_space"), _f32(normals, "normals_image_space")
        isb = is_boundary.detach().to(torch.uint8).contiguous()
        dt = dt.detach().to(torch.uint8).contiguous()
        cr = _f32(crops, "multi_view_crops")
        B, Cn, N = p.shape[0], p.shape[1], p.shape[2]
        U, V = dt.shape[2], dt.shape[3]  # the op takes U = dim 2, V = dim 3
        dev = p.device
        res = torch.empty((B, Cn, N), device=dev)
        res1 = torch.empty((B, Cn, V, U, 2), device=dev)
        dtg = torch.empty((B, Cn, N, 2), device=dev)
        cid = torch.empty((B, Cn, V, U), device=dev)
        P = _lib.ptr
        _lib.call("hc_silhouette_forward", self._h, _stream(), B, Cn, N, U, V, P(p), P(n), P(isb), P(dt), P(cr),
                  P(res), P(res1), P(dtg), P(cid))
        return res, res1, dtg, cid


def silhouette_backward(g, g1, dt_image_grad, closest_vertex_id, crops):
    g, g1 = _f32(g, "mv_dt_grad"), _f32(g1, "mv_dt_grad_1")
    dtg, cid, cr = _f32(dt_image_grad, "dt_image_grad"), _f32(closest_vertex_id, "closest"), _f32(crops, "crops")
    B, Cn, N = g.shape
    V, U = cid.shape[2], cid.shape[3]
    out = torch.empty((B, Cn, N, 2), device=g.device)
    P = _lib.ptr
    _lib.call("hc_silhouette_backward", _stream(), B, Cn, N, U, V, P(g), P(g1), P(dtg), P(cid), P(cr), P(out))
    return out


def silhouette_backward_sized(g, g1, dt_image_grad, closest_vertex_id, crops, widths, heights):
    """Adjoint of ``SilhouetteEngine.forward_sized``: g [B,C,N], g1 [B, pixels, 2]."""
    g, g1 = _f32(g, "mv_dt_grad"), _f32(g1, "mv_dt_grad_1")
    dtg, cid, cr = _f32(dt_image_grad, "dt_image_grad"), _f32(closest_vertex_id, "closest"), _f32(crops, "crops")
    B, Cn, N = g.shape
    w, h = _sizes(widths, heights, Cn)
    out = torch.empty((B, Cn, N, 2), device=g.device)
    P = _lib.ptr
    _lib.call("hc_silhouette_backward_sized", _stream(), B, Cn, N, w.ctypes.data, h.ctypes.data, P(g), P(g1), P(dtg),
              P(cid), P(cr), P(out))
    return out


def _sizes(widths, heights, n):
    """Per-camera image sizes as int32 host arrays [n]."""
    w = np.ascontiguousarray(np.broadcast_to(np.asarray(widths, np.int32), (n,)))
    h = np.ascontiguousarray(np.broadcast_to(np.asarray(heights, np.int32), (n,)))
    return w, h


class _SilFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eng, points, normals, is_boundary, dt, crops):
        res, res1, dtg, cid = eng.forward(points, normals, is_boundary, dt, crops)
        ctx.save_for_backward(dtg, cid, crops)
        ctx.mark_non_differentiable(dtg, cid)
        return res, res1, dtg, cid

    @staticmethod
    def backward(ctx, g, g1, gdtg, gcid):
        dtg, cid, crops = ctx.saved_tensors
        if g is None:
            g = torch.zeros(dtg.shape[:3], device=dtg.device)
        if g1 is None:
            g1 = torch.zeros(tuple(cid.shape) + (2,), device=dtg.device)
        gp = silhouette_backward(g, g1, dtg, cid, crops)
        return None, gp, None, None, None, None


class MultiViewSilhouetteLossGpu:
    """Reference-shaped op: outputs (mv_dt_residual, mv_dt_residual_1, dt_image_gradient, closest_vertex_id)."""

    _engine = None

    def __init__(self, pointsImageSpace, normalsImageSpace, isBoundary, distanceTransformImage, multiViewCrops,
                 engine: SilhouetteEngine | None = None):
        eng = engine or MultiViewSilhouetteLossGpu._default()
        self.multiViewSilhouetteLossGpuOperator = _SilFn.apply(eng, pointsImageSpace, normalsImageSpace, isBoundary,
                                                               distanceTransformImage, multiViewCrops)

    @classmethod
    def _default(cls):
        if cls._engine is None:
            cls._engine = SilhouetteEngine()
        return cls._engine

    def getNode(self):
        return self.multiViewSilhouetteLossGpuOperator
