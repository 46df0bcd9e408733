"""The deform-and-render training step as one object: the composition of
the reference ops that Projects/HoloportedCharacters/HPCMeshDL.py builds in
TF (Pose2EmbeddedGraphCpu -> EmbeddedGraphGpu -> CudaRendererGpu with the L1
image loss, and CameraProjectionGpu -> ProjectedMeshBoundaryGpu ->
MultiViewSilhouetteLossGpu with a sum-of-squares loss on its residuals),
with their registered gradients, issued as C-ABI calls on preallocated
device buffers so that a whole step can be captured in one CUDA graph.

Scene dictionary keys (see ``synthetic.chain_scene``): verts [N,3], faces
[F,3], graph (EmbeddedGraph), markers [8,3], marker_node [8], skeleton,
skin_index / skin_weights [N,K], texcoords, and per-frame dofs [B,D], dT / dA
[B,M,3], disp [B,N,3], colors [B,N,3], texture, sh [B,C,27], extr [B,12C],
intr [B,9C], target [B,C,H,W,3], dt [B,C,H,W] uint8, crops [B,C,7].
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .embedded_graph import EGData, EmbeddedGraphEngine
from .renderer import RendererEngine, _stream
from .silhouette import MeshBoundaryEngine, SilhouetteEngine
from .skinning import Character, SkinningEngine


def character(sc) -> Character:
    return Character.from_synthetic(sc["skeleton"], sc["verts"], sc["faces"], sc["skin_index"])


def eg_data(sc) -> EGData:
    return EGData.from_synthetic(sc["verts"], sc["faces"], sc["graph"], sc["markers"], sc["marker_node"])


class DeformRenderChain:
    """One fwd + loss + bwd step of the deform-and-render chain through
    libhc.so on device-resident buffers:

      dofs -> node skinning (Pose2EG) -> EG deformation -> raster (vertexColor)
           -> masked L1 image loss
      EG vertices -> camera projection -> mesh boundary -> silhouette DT loss
      adjoints back to node rotations / translations and vertex colours.

    ``deformation="dq"`` replaces node skinning + EG by per-vertex dual-
    quaternion skinning of the character (DqSkinningGpu), the composition of
    a skinned character without an embedded graph; its adjoint carries the
    vertex gradient to the joint angles.  ``width`` / ``height`` may be
    per-camera sequences: cameras of different sizes share every call, and
    the per-pixel buffers are [B, pixels of a frame, ...] with the frame's
    cameras concatenated in order (the reference needs one op per size).

    ``loss`` holds (L1, silhouette model->data, silhouette data->model);
    ``buf`` holds every intermediate and gradient (``gT`` / ``gA`` are the
    node translation / rotation gradients, ``gcol`` the vertex colours',
    ``gdofs`` the joint angles' when ``joint_gradients`` is set: the EG then
    returns its skinned-transform gradients and the node skinning's adjoint
    carries them to the dofs; the reference chain has no such gradient, its
    Pose2EmbeddedGraphCpu op being non-differentiable)."""

    def __init__(self, sc, dev, frames: int, views: int, width, height, w_sil: float = 1e-3,
                 w_sil1: float = 1e-3, tile: int = 8, bin_capacity: int = 256, gradient_parity: bool = False,
                 joint_gradients: bool = True, fused_l1: bool = True, deformation: str = "eg"):
        B, C, N = frames, views, int(sc["verts"].shape[0])
        # one image size for all cameras, or one per camera (`width` / `height`
        # sequences): then every per-pixel buffer is [B, pixels of a frame, ...]
        # with the frame's cameras concatenated, and one call still covers all views
        ws = np.ascontiguousarray(np.broadcast_to(np.asarray(width, np.int32), (C,)))
        hs = np.ascontiguousarray(np.broadcast_to(np.asarray(height, np.int32), (C,)))
        self.widths, self.heights = ws, hs
        self.multires = not (np.all(ws == ws[0]) and np.all(hs == hs[0]))
        W, H = int(ws[0]), int(hs[0])
        self.P_frame = int((ws.astype(np.int64) * hs).sum())
        if deformation not in ("eg", "dq"):
            raise ValueError("deformation must be 'eg' (node skinning + embedded graph) or 'dq' (vertex DQ skinning)")
        self.deformation = deformation
        M = int(sc["graph"].n_nodes) if deformation == "eg" else 0
        Mk = int(len(sc["markers"])) if deformation == "eg" else 0
        self.B, self.C, self.H, self.W, self.N, self.M, self.Mk = B, C, H, W, N, M, Mk
        self.w_sil, self.w_sil1 = float(w_sil), float(w_sil1)
        self.skin = SkinningEngine(character(sc))
        self.skin.reserve(B)
        self.joint_gradients = bool(joint_gradients)
        # the image L1 inside the raster's tile pass and adjoint
        # (hc_renderer_forward_l1 / _backward_l1) or as its own op
        # (hc_image_l1_loss + hc_renderer_backward on the gradient image)
        self.fused_l1 = bool(fused_l1)
        if deformation == "eg":
            self.eg = EmbeddedGraphEngine(eg_data(sc), full_skinned_gradient=self.joint_gradients)
            self.eg.reserve(B)
        self.rend = RendererEngine(sc["faces"], sc["texcoords"], N, C, ws if self.multires else W,
                                   hs if self.multires else H, "vertexColor", "shadeless", 2, 2)
        self.rend.set_tuning(tile, bin_capacity)
        self.tuning = (tile, bin_capacity)
        if gradient_parity:
            _lib.call("hc_renderer_set_gradient_parity", self.rend.handle, 1)
        self.rend.reserve(B)
        self.mb = MeshBoundaryEngine(sc["faces"], N)
        self.sil = SilhouetteEngine()
        if self.multires:
            self.mb.reserve_sized(B, C, ws, hs)
            self.sil.reserve_sized(B, C, N, ws, hs)
        else:
            self.mb.reserve(B, C, W, H)
            self.sil.reserve(B, C, N, W, H)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        keys = ("dofs", "dT", "dA", "disp", "colors", "texture", "sh", "extr", "intr", "target", "dt", "crops")
        self.inp = {k: t(sc[k]) for k in keys if k in sc}
        self.tex_hw = (int(sc["texture"].shape[1]), int(sc["texture"].shape[2]))
        self.skin_w = t(np.asarray(sc["skin_weights"], np.float32))
        e = lambda *shape, dt=torch.float32: torch.empty(shape, device=dev, dtype=dt)  # noqa: E731
        img = (B, self.P_frame) if self.multires else (B, C, H, W)
        self.buf = dict(
            v=e(B, N, 3), n=e(B, N, 3),
            bary=e(*img, 2), face=e(*img, dt=torch.int32), render=e(*img, 3),
            vnormal=e(B, C, N, 3), grad_img=None if fused_l1 else e(*img, 3),
            p2d=e(B, C, N, 2), n2d=e(B, C, N, 2), isb=e(B, C, N, dt=torch.uint8),
            res=e(B, C, N), res1=e(*img, 2), dtg=e(B, C, N, 2), cid=e(*img),
            g_res=e(B, C, N), gp2d=e(B, C, N, 2), gv_sil=e(B, N, 3),
            gv=e(B, N, 3), gcol=e(B, N, 3), gsh=e(B, C, 27),
            gdofs=torch.zeros((B, self.skin.D), device=dev))
        if deformation == "eg":
            self.node_vertex = t(sc["graph"].node_vertex.astype(np.int32))
            self.buf.update(sT=e(B, M, 3), sA=e(B, M, 3), dq=e(B, self.skin.S, 8), mk=e(B, Mk, 3),
                            graph=e(B, M, 3), da=e(B, M, 3), sa=e(B, M, 3), gm=torch.zeros((B, Mk, 3), device=dev),
                            gT=e(B, M, 3), gA=e(B, M, 3), gsT=e(B, M, 3), gsA=e(B, M, 3), gdisp=e(B, N, 3))
        else:  # per-vertex DQ skinning: the frame's skin weights, joints and dual quaternions
            K = self.skin.K
            self.buf.update(weights=self.skin_w.unsqueeze(0).expand(B, N, K).contiguous(), gjp=e(B, self.skin.J, 3),
                            gja=e(B, self.skin.J, 3), dq=e(B, self.skin.S, 8), outw=e(B, N, K), gw=e(B, N, K))
        self.loss = torch.zeros((3,), device=dev)
        # the stream of the silhouette branch (step), and the adjoint's static
        # tile schedule, under which CTAs that run out early make room for it
        self._side = torch.cuda.Stream(device=self.loss.device) if self.loss.is_cuda else None
        if self._side is not None:
            _lib.call("hc_renderer_set_adjoint_schedule", self.rend.handle, 0)
        self.ws = torch.zeros((8,), device=dev, dtype=torch.float64)

    def forward(self):
        """Deformation (node skinning + EG, or vertex DQ skinning), raster and the
        L1 image loss + its gradient."""
        L, P, s = _lib.call, _lib.ptr, _stream()
        i, o = self.inp, self.buf
        B, C, M = self.B, self.C, self.M
        if self.deformation == "eg":
            L("hc_pose2eg_forward", self.skin.handle, s, B, P(i["dofs"]), M, P(self.node_vertex), P(self.skin_w),
              P(o["sT"]), P(o["sA"]), P(o["dq"]))
            L("hc_eg_forward", self.eg.handle, s, B, P(i["dT"]), P(i["dA"]), P(o["sT"]), P(o["sA"]), P(i["disp"]),
              P(o["v"]), P(o["n"]), P(o["mk"]), P(o["graph"]), P(o["da"]), P(o["sa"]))
        else:
            L("hc_dq_skinning_forward", self.skin.handle, s, B, P(i["dofs"]), P(o["weights"]), P(o["v"]), P(o["n"]),
              P(o["gjp"]), P(o["gja"]), P(o["dq"]), P(o["outw"]))
        if self.fused_l1:
            L("hc_renderer_forward_l1", self.rend.handle, s, B, P(o["v"]), P(i["colors"]), P(i["texture"]),
              *self.tex_hw, P(i["sh"]), P(i["extr"]), P(i["intr"]), P(o["bary"]), P(o["face"]), P(o["render"]),
              P(o["vnormal"]), P(i["target"]), None, P(self.ws), P(self.loss))
            return
        L("hc_renderer_forward", self.rend.handle, s, B, P(o["v"]), P(i["colors"]), P(i["texture"]), *self.tex_hw,
          P(i["sh"]), P(i["extr"]), P(i["intr"]), P(o["bary"]), P(o["face"]), P(o["render"]), P(o["vnormal"]), None)
        L("hc_image_l1_loss", s, B * self.P_frame, P(o["render"]), P(i["target"]), P(o["face"]), None, P(self.ws),
          P(self.loss), P(o["grad_img"]))

    def silhouette_forward(self):
        """Camera projection, mesh boundary, silhouette DT loss + residual gradients."""
        L, P, s = _lib.call, _lib.ptr, _stream()
        i, o = self.inp, self.buf
        B, C, H, W, N = self.B, self.C, self.H, self.W, self.N
        L("hc_camera_projection_forward", s, B, C, N, P(o["v"]), None, P(i["extr"]), P(i["intr"]), 1, P(o["p2d"]))
        L("hc_camera_projection_forward", s, B, C, N, P(o["v"]), P(o["n"]), P(i["extr"]), P(i["intr"]), 0,
          P(o["n2d"]))
        # the renderer's face buffer of the same views is the coverage hint
        ws, hs = self.widths.ctypes.data, self.heights.ctypes.data
        if self.multires:
            L("hc_mesh_boundary_forward_sized", self.mb.handle, s, B, C, ws, hs, P(o["v"]), P(i["extr"]),
              P(i["intr"]), P(o["p2d"]), P(o["face"]), P(o["isb"]))
        else:
            L("hc_mesh_boundary_forward_hinted", self.mb.handle, s, B, C, W, H, P(o["v"]), P(i["extr"]),
              P(i["intr"]), P(o["p2d"]), P(o["face"]), P(o["isb"]))
        # the per-pixel residual's squared loss is formed inside the silhouette
        # forward (the residual is non-zero only on the target's silhouette),
        # and its adjoint reads the residual itself (silhouette_backward)
        L("hc_silhouette_forward_sumsq_sized", self.sil.handle, s, B, C, N, ws, hs, P(o["p2d"]), P(o["n2d"]),
          P(o["isb"]), P(i["dt"]), P(i["crops"]), P(o["res"]), P(o["res1"]), P(o["dtg"]), P(o["cid"]),
          self.w_sil1, self.ws.data_ptr() + 24, self.loss.data_ptr() + 8)
        L("hc_sum_squares_loss", s, B * C * N, P(o["res"]), self.w_sil, self.ws.data_ptr() + 16,
          self.loss.data_ptr() + 4, P(o["g_res"]))

    def silhouette_backward(self):
        """Silhouette adjoint and the camera-projection adjoint to vertex positions."""
        L, P, s = _lib.call, _lib.ptr, _stream()
        i, o = self.inp, self.buf
        B, C, H, W, N = self.B, self.C, self.H, self.W, self.N
        # d (w1 sum res1^2) / d res1 = 2 w1 res1, applied to the residual as it is read
        L("hc_silhouette_backward_scaled_sized", s, B, C, N, self.widths.ctypes.data, self.heights.ctypes.data,
          P(o["g_res"]), P(o["res1"]), 2.0 * self.w_sil1, P(o["dtg"]), P(o["cid"]), P(i["crops"]), P(o["gp2d"]))
        L("hc_camera_projection_backward", s, B, C, N, P(o["gp2d"]), P(o["v"]), P(i["extr"]), P(i["intr"]), 1,
          P(o["gv_sil"]))

    def backward(self, join=None):
        """Raster adjoint, the sum of the two vertex-position gradients, then the
        deformation's adjoint: EG (and the node-skinning adjoint to the joint
        angles), or the vertex DQ skinning's to the joint angles.  ``join``: a
        stream whose work (the silhouette branch) the sum waits for."""
        L, P, s = _lib.call, _lib.ptr, _stream()
        i, o = self.inp, self.buf
        B, N = self.B, self.N
        if self.fused_l1:
            L("hc_renderer_backward_l1", self.rend.handle, s, B, P(self.ws), P(o["render"]), None, P(o["v"]),
              P(i["colors"]), P(i["texture"]), *self.tex_hw, P(i["sh"]), P(i["target"]), P(o["vnormal"]),
              P(o["bary"]), P(o["face"]), P(i["extr"]), P(i["intr"]), P(o["gv"]), P(o["gcol"]), None, P(o["gsh"]))
        else:
            L("hc_renderer_backward", self.rend.handle, s, B, P(o["grad_img"]), P(o["v"]), P(i["colors"]),
              P(i["texture"]), *self.tex_hw, P(i["sh"]), P(i["target"]), P(o["vnormal"]), P(o["bary"]),
              P(o["face"]), P(i["extr"]), P(i["intr"]), P(o["gv"]), P(o["gcol"]), None, P(o["gsh"]))
        if join is not None:
            torch.cuda.current_stream().wait_stream(join)
        L("hc_add_inplace", s, B * N * 3, P(o["gv"]), P(o["gv_sil"]))
        if self.deformation == "dq":  # joint angles (and skin weights) through the vertex DQ skinning
            L("hc_dq_skinning_backward", self.skin.handle, s, B, P(o["gv"]), P(o["v"]), P(o["gjp"]), P(o["gja"]),
              P(o["dq"]), P(o["weights"]), P(o["gdofs"]), P(o["gw"]))
            return
        full = self.joint_gradients
        L("hc_eg_backward", self.eg.handle, s, B, P(o["gv"]), P(o["gm"]), P(o["da"]), P(o["sa"]), P(o["gT"]),
          P(o["gA"]), P(o["gsT"]), P(o["gsA"]), P(o["gdisp"]), P(i["dT"]) if full else None,
          P(i["disp"]) if full else None)
        if full:  # joint angles through the node skinning
            L("hc_pose2eg_backward", self.skin.handle, s, B, P(i["dofs"]), self.M, P(self.node_vertex),
              P(self.skin_w), P(o["gsT"]), P(o["gsA"]), P(o["gdofs"]))

    def autotune(self, candidates=((8, 128), (8, 256), (8, 512), (8, 1024), (16, 256), (16, 512), (16, 1024),
                                   (32, 512), (32, 1024)), reps: int = 3):
        """Pick the raster's bin-tile size and bin capacity by timing the
        forward stage on the current inputs (CUDA events, after a warm-up
        call per candidate); candidates whose spill capacity overflows are
        skipped.  Sets the fastest and returns {(tile, cap): ms}."""
        results = {}
        for tile, cap in candidates:
            self.rend.set_tuning(tile, cap)
            self.rend.reserve(self.B)
            try:
                self.forward()
                self.rend.stats()
            except _lib.HcError:
                continue
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                self.forward()
            b.record()
            torch.cuda.synchronize()
            results[(tile, cap)] = a.elapsed_time(b) / reps
        best = min(results, key=results.get)
        self.rend.set_tuning(*best)
        self.rend.reserve(self.B)
        self.tuning = best
        return results

    def check(self):
        """Run the forward stage once and raise if the raster's spill
        capacity overflowed (the result would be incomplete); returns
        (binned, spilled) pair counts."""
        self.forward()
        return self.rend.stats()

    def step(self):
        """One training step.  After the forward stage the silhouette branch
        (boundary, loss and its adjoint) and the raster adjoint are independent
        until their vertex-position gradients are summed, so the silhouette
        branch runs on a second stream beside the raster adjoint (its kernels
        wait on gathers and leave issue slots that the adjoint uses), joined
        before the sum; a captured graph keeps the two branches."""
        self.forward()
        if self.loss.is_cuda:
            self._side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(self._side):
                self.silhouette_forward()
                self.silhouette_backward()
            self.backward(join=self._side)
        else:
            self.silhouette_forward()
            self.silhouette_backward()
            self.backward()

    def capture_step(self, inputs: dict | None = None) -> torch.cuda.CUDAGraph:
        """Capture one step (forward, silhouette, both adjoints) in a CUDA
        graph that reads the tensors of ``inputs`` (keys and shapes of
        ``self.inp``; the current inputs by default).  A replay runs the step
        on what those tensors hold at that time.  Run one eager step first: it
        sizes every workspace, and no allocation may happen during capture."""
        saved = dict(self.inp)
        if inputs:
            for k, v in inputs.items():
                if k not in self.inp or v.shape != self.inp[k].shape or v.dtype != self.inp[k].dtype:
                    raise ValueError(f"input {k!r} must match the chain's {k} tensor")
            self.inp.update(inputs)
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream(device=self.loss.device)
        s.wait_stream(torch.cuda.current_stream())
        try:
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    self.step()
        finally:
            torch.cuda.current_stream().wait_stream(s)
            self.inp.clear()
            self.inp.update(saved)
        return g

    def stages(self):
        return (("deform_render_forward", self.forward), ("silhouette_forward", self.silhouette_forward),
                ("silhouette_backward", self.silhouette_backward), ("render_eg_backward", self.backward))
