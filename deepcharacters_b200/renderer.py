"""Differentiable multi-view rasterizer: drop-in for ``CudaRendererGpu``.

Mirrors the reference Python class (Projects/CudaRenderer/CudaRendererGPU.py:25-237)
and its op attributes (CudaRenderer/cpp/src/TensorflowOperators/CudaRenderer/
CudaRenderer.cpp:5-31): same constructor arguments, same outputs and
getters, same gradient rule (only ``vertexColor`` and ``textured`` -- and the
added ``texturedBilinear`` -- produce
gradients; target image and cameras always get zeros).  Tensors are torch
CUDA tensors; the work runs in ``libhc.so`` on the current CUDA stream.
"""
from __future__ import annotations

import ctypes as C
import functools

import numpy as np
import torch

from . import _lib

ALBEDO_MODES = ("vertexColor", "textured", "normal", "lighting", "foregroundMask", "position", "depth", "uv",
                "texturedBilinear")  # the last: bilinear texture sampling, no reference counterpart
SHADING_MODES = ("shaded", "shadeless")
NORMAL_MAP_MODES = ("none", "normal", "position", "face")


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def _f32(t: torch.Tensor | None, name: str) -> torch.Tensor | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    return t.detach().to(torch.float32).contiguous()


class RendererEngine:
    """Owns one ``hc_renderer`` handle (topology, camera rig, modes, workspace)."""

    def __init__(self, faces, tex_coords, n_vertices: int, n_cameras: int, width: int, height: int,
                 albedo_mode: str = "textured", shading_mode: str = "shaded", image_filter_size: int = 1,
                 texture_filter_size: int = 1, compute_normal_map: str = "none"):
        f = np.ascontiguousarray(np.asarray(faces, dtype=np.int32).reshape(-1))
        tc = None if tex_coords is None or len(tex_coords) == 0 else np.ascontiguousarray(
            np.asarray(tex_coords, dtype=np.float32).reshape(-1))
        if f.size % 3:
            raise ValueError("No triangular faces!")
        self.F = f.size // 3
        self.N = int(n_vertices)
        self.C = int(n_cameras)
        # width / height: one size for all cameras, or one per camera (views of
        # different sizes then share one launch; image buffers are flat
        # [B, pixels of a frame, ...] with the frame's cameras concatenated)
        ws = np.broadcast_to(np.asarray(width, np.int32), (self.C,)).copy()
        hs = np.broadcast_to(np.asarray(height, np.int32), (self.C,)).copy()
        self.multires = not (np.all(ws == ws[0]) and np.all(hs == hs[0]))
        self.widths, self.heights = ws, hs
        self.W = int(ws[0])
        self.H = int(hs[0])
        self.P_frame = int((ws.astype(np.int64) * hs).sum())
        self.albedo_mode = albedo_mode
        self.shading_mode = shading_mode
        self.image_filter_size = int(image_filter_size)
        self.texture_filter_size = int(texture_filter_size)
        self.compute_normal_map = compute_normal_map
        self.faces = f
        self.tex_coords = tc
        h = C.c_void_p()
        if self.multires:
            _lib.call("hc_renderer_create_multires", C.byref(h), f.ctypes.data, self.F,
                      None if tc is None else tc.ctypes.data, 0 if tc is None else tc.size, self.N, self.C,
                      ws.ctypes.data, hs.ctypes.data, albedo_mode.encode(), shading_mode.encode(),
                      self.image_filter_size, self.texture_filter_size, compute_normal_map.encode())
        else:
            _lib.call("hc_renderer_create", C.byref(h), f.ctypes.data, self.F,
                      None if tc is None else tc.ctypes.data, 0 if tc is None else tc.size,
                      self.N, self.C, self.W, self.H, albedo_mode.encode(), shading_mode.encode(),
                      self.image_filter_size, self.texture_filter_size, compute_normal_map.encode())
        self._h = h

    def image_shape(self, B: int) -> tuple:
        """Leading shape of the per-pixel buffers: [B, C, H, W] or, with
        per-camera sizes, [B, pixels of a frame]."""
        return (B, self.P_frame) if self.multires else (B, self.C, self.H, self.W)

    def split_views(self, img: torch.Tensor) -> list:
        """[B, P_frame, ...] buffer -> per camera [B, H_c, W_c, ...] views (no copy)."""
        out, o = [], 0
        for w, h in zip(self.widths, self.heights):
            n = int(w) * int(h)
            out.append(img[:, o:o + n].reshape((img.shape[0], int(h), int(w)) + tuple(img.shape[2:])))
            o += n
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib.lib().hc_renderer_destroy(h)
            self._h = None

    KERNELS = ("view_setup", "vertex_normals", "tri_frame", "bin", "spill", "resolve", "render_grad",
               "normal_chain")

    def set_kernel_timing(self, enable: bool):
        """Bracket every renderer launch with CUDA events (benchmarks only)."""
        _lib.call("hc_renderer_set_kernel_timing", self._h, int(bool(enable)))

    def kernel_times(self) -> dict:
        """Last recorded duration (ms) of each renderer kernel since the previous read."""
        import ctypes as _C
        out = (_C.c_float * len(self.KERNELS))()
        _lib.call("hc_renderer_kernel_times", self._h, _C.cast(out, _C.c_void_p), len(self.KERNELS))
        return {k: float(v) for k, v in zip(self.KERNELS, out) if v >= 0}

    @property
    def handle(self):
        return self._h

    def reserve(self, batch: int):
        _lib.call("hc_renderer_reserve", self._h, int(batch))

    def set_tuning(self, tile: int, bin_capacity: int):
        _lib.call("hc_renderer_set_tuning", self._h, int(tile), int(bin_capacity))

    def set_gradient_parity(self, parity: bool):
        """True: the reference's barycentric-Jacobian formula; False (default): exact closed form."""
        _lib.call("hc_renderer_set_gradient_parity", self._h, int(bool(parity)))

    def set_adjoint_schedule(self, dynamic: bool):
        """True (default): the adjoint's CTAs claim tiles from a counter; False:
        a fixed tile stride per CTA (leaves SMs free early for work running
        concurrently on another stream).  Same results either way."""
        _lib.call("hc_renderer_set_adjoint_schedule", self._h, int(bool(dynamic)))

    def stats(self) -> tuple[int, int]:
        b = C.c_int64()
        s = C.c_int64()
        _lib.call("hc_renderer_stats", self._h, _stream(), C.byref(b), C.byref(s))
        return b.value, s.value

    def forward(self, vertex_pos, vertex_color, texture, sh_coeff, extrinsics, intrinsics, batch: int | None = None,
                diagnostics: bool = False, out: dict | None = None):
        """Raw forward.  Returns (bary, face, render, vertex_normal, normal_map[, depth_q, tie_count])."""
        vp = _f32(vertex_pos, "vertex_pos")
        B = int(batch if batch is not None else vp.shape[0])
        dev = vp.device
        vc = _f32(vertex_color, "vertex_color")
        tex = _f32(texture, "texture")
        sh = _f32(sh_coeff, "sh_coeff")
        ex = _f32(extrinsics, "extrinsics")
        it = _f32(intrinsics, "intrinsics")
        TH = int(tex.shape[1]) if tex is not None and tex.dim() == 4 else 0
        TW = int(tex.shape[2]) if tex is not None and tex.dim() == 4 else 0
        o = out or {}
        img = self.image_shape(B)
        bary = o.get("bary") if o.get("bary") is not None else torch.empty(
            img + (2,), device=dev, dtype=torch.float32)
        face = o.get("face") if o.get("face") is not None else torch.empty(img, device=dev, dtype=torch.int32)
        render = o.get("render") if o.get("render") is not None else torch.empty(
            img + (3,), device=dev, dtype=torch.float32)
        vnormal = o.get("vnormal") if o.get("vnormal") is not None else torch.empty(
            (B, self.C, self.N, 3), device=dev, dtype=torch.float32)
        normal_map = torch.zeros((B, max(TH, 1), max(TW, 1), 3), device=dev, dtype=torch.float32)
        depth_q = tie = None
        if diagnostics:
            depth_q = torch.empty(img, device=dev, dtype=torch.int32)
            tie = torch.empty(img, device=dev, dtype=torch.int32)
        P = _lib.ptr
        _lib.call("hc_renderer_forward_ex", self._h, _stream(), B, P(vp), P(vc), P(tex), TH, TW, P(sh), P(ex), P(it),
                  P(bary), P(face), P(render), P(vnormal),
                  P(normal_map) if self.compute_normal_map != "none" else None, P(depth_q), P(tie))
        res = (bary, face, render, vnormal, normal_map)
        if diagnostics:
            res = res + (depth_q, tie)
        return res


@functools.lru_cache(maxsize=16)
def _engine_cached(key):
    (faces, tc, N, Cn, W, H, am, sm, ifs, tfs, nm) = key
    return RendererEngine(np.frombuffer(faces, np.int32), None if tc is None else np.frombuffer(tc, np.float32),
                          N, Cn, W, H, am, sm, ifs, tfs, nm)


def get_engine(faces, tex_coords, n_vertices, n_cameras, width, height, albedo_mode, shading_mode,
               image_filter_size, texture_filter_size, compute_normal_map) -> RendererEngine:
    """Engine per attribute set, like one TF op instance per graph node."""
    f = np.ascontiguousarray(np.asarray(faces, dtype=np.int32).reshape(-1)).tobytes()
    tc = None if tex_coords is None or len(tex_coords) == 0 else np.ascontiguousarray(
        np.asarray(tex_coords, dtype=np.float32).reshape(-1)).tobytes()
    return _engine_cached((f, tc, int(n_vertices), int(n_cameras), int(width), int(height), albedo_mode,
                           shading_mode, int(image_filter_size), int(texture_filter_size), compute_normal_map))


class _RenderFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, engine: RendererEngine, vertex_pos, vertex_color, texture, sh_coeff, target_image,
                extrinsics, intrinsics):
        # batch size comes from the texture, as in CudaRenderer.cpp:233
        B = int(texture.shape[0])
        bary, face, render, vnormal, normal_map = engine.forward(vertex_pos, vertex_color, texture, sh_coeff,
                                                                 extrinsics, intrinsics, batch=B)
        ctx.engine = engine
        ctx.save_for_backward(vertex_pos, vertex_color, texture, sh_coeff, target_image, extrinsics, intrinsics,
                              bary, face, vnormal)
        ctx.mark_non_differentiable(face)
        return bary, face, render, vnormal, normal_map

    @staticmethod
    def backward(ctx, g_bary, g_face, g_render, g_vnormal, g_normal_map):
        (vertex_pos, vertex_color, texture, sh_coeff, target_image, extrinsics, intrinsics, bary, face,
         vnormal) = ctx.saved_tensors
        eng: RendererEngine = ctx.engine
        zeros = [torch.zeros_like(t) if t is not None else None
                 for t in (vertex_pos, vertex_color, texture, sh_coeff)]
        if eng.albedo_mode in ("vertexColor", "textured", "texturedBilinear") and g_render is not None:
            grads = renderer_backward(eng, g_render, vertex_pos, vertex_color, texture, sh_coeff, target_image,
                                      vnormal, bary, face, extrinsics, intrinsics)
        else:
            grads = zeros
        return (None, grads[0], grads[1], grads[2], grads[3], torch.zeros_like(target_image),
                torch.zeros_like(extrinsics), torch.zeros_like(intrinsics))


def renderer_backward(engine: RendererEngine, render_buffer_grad, vertex_pos, vertex_color, texture, sh_coeff,
                      target_image, vertex_normal, barycentric_buffer, face_buffer, extrinsics, intrinsics,
                      batch: int | None = None):
    """``CudaRendererGradGpu``: gradients w.r.t. vertex_pos, vertex_color, texture, sh_coeff.

    The batch size comes from ``vertex_pos`` (CudaRendererGrad.cpp:184)."""
    vp = _f32(vertex_pos, "vertex_pos")
    B = int(batch if batch is not None else vp.shape[0])
    dev = vp.device
    g = _f32(render_buffer_grad, "render_buffer_grad")
    vc = _f32(vertex_color, "vertex_color")
    tex = _f32(texture, "texture")
    sh = _f32(sh_coeff, "sh_coeff")
    tgt = _f32(target_image, "target_image")
    vn = _f32(vertex_normal, "vertex_normal")
    bary = _f32(barycentric_buffer, "barycentric_buffer")
    face = face_buffer.detach().to(torch.int32).contiguous()
    ex = _f32(extrinsics, "extrinsics")
    it = _f32(intrinsics, "intrinsics")
    TH = int(tex.shape[1]) if tex is not None and tex.dim() == 4 else 0
    TW = int(tex.shape[2]) if tex is not None and tex.dim() == 4 else 0
    gpos = torch.empty((B, engine.N, 3), device=dev, dtype=torch.float32)
    gcol = torch.zeros((B, engine.N, 3), device=dev, dtype=torch.float32)
    gtex = torch.zeros((B, max(TH, 1), max(TW, 1), 3), device=dev, dtype=torch.float32)
    gsh = torch.zeros((B, engine.C, 27), device=dev, dtype=torch.float32)
    P = _lib.ptr
    _lib.call("hc_renderer_backward", engine.handle, _stream(), B, P(g), P(vp), P(vc), P(tex), TH, TW, P(sh), P(tgt),
              P(vn), P(bary), P(face), P(ex), P(it), P(gpos), P(gcol), P(gtex) if TH > 0 else None, P(gsh))
    return gpos, gcol, gtex, gsh


class CudaRendererGpu:
    """Reference-shaped wrapper (Projects/CudaRenderer/CudaRendererGPU.py:25-188)."""

    def __init__(self, faces_attr=(), texCoords_attr=(), numberOfVertices_attr=-1, numberOfCameras_attr=-1,
                 renderResolutionU_attr=-1, renderResolutionV_attr=-1, albedoMode_attr="textured",
                 shadingMode_attr="shaded", image_filter_size_attr=1, texture_filter_size_attr=1,
                 compute_normal_map_attr="none", vertexPos_input=None, vertexColor_input=None,
                 texture_input=None, shCoeff_input=None, targetImage_input=None, extrinsics_input=(),
                 intrinsics_input=(), nodeName="CudaRenderer"):
        self.faces_attr = faces_attr
        self.texCoords_attr = texCoords_attr
        self.numberOfVertices_attr = numberOfVertices_attr
        self.numberOfCameras_attr = numberOfCameras_attr
        self.renderResolutionU_attr = renderResolutionU_attr
        self.renderResolutionV_attr = renderResolutionV_attr
        self.albedoMode_attr = albedoMode_attr
        self.shadingMode_attr = shadingMode_attr
        self.image_filter_size_attr = image_filter_size_attr
        self.texture_filter_size_attr = texture_filter_size_attr
        self.compute_normal_map_attr = compute_normal_map_attr
        self.vertexPos_input = vertexPos_input
        self.vertexColor_input = vertexColor_input
        self.texture_input = texture_input
        self.shCoeff_input = shCoeff_input
        self.targetImage_input = targetImage_input
        self.extrinsics_input = extrinsics_input
        self.intrinsics_input = intrinsics_input
        self.nodeName = nodeName
        self.engine = get_engine(faces_attr, texCoords_attr, numberOfVertices_attr, numberOfCameras_attr,
                                 renderResolutionU_attr, renderResolutionV_attr, albedoMode_attr, shadingMode_attr,
                                 image_filter_size_attr, texture_filter_size_attr, compute_normal_map_attr)
        self.cudaRendererOperator = _RenderFn.apply(self.engine, vertexPos_input, vertexColor_input, texture_input,
                                                    shCoeff_input, targetImage_input, extrinsics_input,
                                                    intrinsics_input)

    def getBaryCentricBufferTF(self):
        return self.cudaRendererOperator[0]

    def getFaceBufferTF(self):
        return self.cudaRendererOperator[1]

    def getVertexNormalTF(self):
        return self.cudaRendererOperator[3]

    def getRenderBufferTF(self):
        return self.cudaRendererOperator[2]

    def getNormalMap(self):
        if self.compute_normal_map_attr and self.compute_normal_map_attr != "none":
            return self.cudaRendererOperator[4].reshape(self.texture_input.shape)
        return None

    def getModelMaskTF(self):
        face = self.cudaRendererOperator[1]
        return (face >= 0).unsqueeze(-1).expand(*face.shape, 3).to(torch.float32)
