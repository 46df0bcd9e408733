"""Dual-quaternion and linear-blend skinning with device forward kinematics.

Drop-in for the ``DqSkinningGpu`` / ``LbSkinningGpu`` ops and their gradient
ops (CustomTensorFlowCPPOperators/src/CustomGPUOperators/DQSkinningOperator/
DQSkinningGPUOp.cpp:5-15, DQSkinningGPUOpGrad.cpp:5-15; LBSkinningOperator/
LBSkinningGPUOp.cpp:5-16, LBSkinningGPUOpGrad.cpp:5-16): same inputs
(dofs, skinning weights, displacements), same six outputs and the same
gradient outputs.  The reference builds the character from files and runs
forward kinematics on the host in every call; here the character arrays are
passed once (``Character``) and the kinematics run on the device.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np
import torch

from . import _lib
from .renderer import _f32, _stream

REVOLUTE, PRISMATIC = 0, 1


@dataclasses.dataclass
class Character:
    """Skeleton + skinned mesh arrays (what the .character/.skeleton/.skin loaders produce)."""
    parent: np.ndarray          # [J] int32, -1 root, parents first
    joint_type: np.ndarray      # [J] int32 (0 revolute, 1 prismatic)
    offset: np.ndarray          # [J,3] mm
    axis: np.ndarray            # [J,3]
    dof_offsets: np.ndarray     # [D+1]
    dof_joint: np.ndarray       # [E]
    dof_weight: np.ndarray      # [E]
    skin_joint: np.ndarray      # [S]
    base_vertices: np.ndarray   # [N,3]
    base_normals: np.ndarray    # [N,3]
    skin_index: np.ndarray      # [N,K]
    joint_scale: np.ndarray | None = None
    skin_scale: np.ndarray | None = None

    @property
    def n_joints(self):
        return int(self.parent.shape[0])

    @property
    def n_dofs(self):
        return int(self.dof_offsets.shape[0] - 1)

    @property
    def n_skin(self):
        return int(self.skin_joint.shape[0])

    @classmethod
    def from_synthetic(cls, skel, verts, faces, skin_index):
        v = np.asarray(verts, np.float64)
        n = np.zeros_like(v)
        f = np.asarray(faces)
        fn = np.cross(v[f[:, 1]] - v[f[:, 0]], v[f[:, 2]] - v[f[:, 0]])
        for k in range(3):
            np.add.at(n, f[:, k], fn)
        n /= np.linalg.norm(n, axis=1, keepdims=True)
        D = skel.n_dofs
        return cls(skel.parent.astype(np.int32), np.zeros(skel.n_joints, np.int32), skel.offset.astype(np.float32),
                   skel.axis.astype(np.float32), np.arange(D + 1, dtype=np.int32), skel.dof_joint.astype(np.int32),
                   skel.dof_weight.astype(np.float32), skel.skin_joint.astype(np.int32), v.astype(np.float32),
                   n.astype(np.float32), np.asarray(skin_index, np.int32))


class SkinningEngine:
    """Owns one ``hc_skin`` handle."""

    def __init__(self, ch: Character, parity: bool = True):
        a = lambda x, dt: None if x is None else np.ascontiguousarray(np.asarray(x, dt))  # noqa: E731
        self._k = dict(parent=a(ch.parent, np.int32), type=a(ch.joint_type, np.int32), offset=a(ch.offset, np.float32),
                       axis=a(ch.axis, np.float32), js=a(ch.joint_scale, np.float32),
                       doff=a(ch.dof_offsets, np.int32), dj=a(ch.dof_joint, np.int32), dw=a(ch.dof_weight, np.float32),
                       sj=a(ch.skin_joint, np.int32), ss=a(ch.skin_scale, np.float32),
                       bv=a(ch.base_vertices, np.float32), bn=a(ch.base_normals, np.float32),
                       si=a(ch.skin_index, np.int32))
        k = self._k
        self.J, self.D, self.S = ch.n_joints, ch.n_dofs, ch.n_skin
        self.N, self.K = k["si"].shape
        h = C.c_void_p()
        P = _lib.ptr
        _lib.call("hc_skin_create", C.byref(h), self.J, P(k["parent"]), P(k["type"]), P(k["offset"]), P(k["axis"]),
                  P(k["js"]), self.D, P(k["doff"]), P(k["dj"]), P(k["dw"]), self.S, P(k["sj"]), P(k["ss"]), self.N,
                  P(k["bv"]), P(k["bn"]), self.K, P(k["si"]))
        self._h = h
        self.set_parity(parity)

    @classmethod
    def from_file(cls, character_file_path: str, parity: bool = True) -> "SkinningEngine":
        """The op's construction from ``character_file_path_skinning`` (DQSkinningGPUOp.cpp:22-44)."""
        from . import loaders
        return cls(loaders.load_character(character_file_path).character(), parity)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib.lib().hc_skin_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def set_parity(self, parity: bool):
        self.parity = bool(parity)
        _lib.call("hc_skin_set_parity", self._h, int(self.parity))

    def reserve(self, batch: int):
        _lib.call("hc_skin_reserve", self._h, int(batch))

    def _outs(self, B, dev, last):
        e = lambda *s: torch.empty(s, device=dev)  # noqa: E731
        return (e(B, self.N, 3), e(B, self.N, 3), e(B, self.J, 3), e(B, self.J, 3), e(B, self.S, last),
                e(B, self.N, self.K))

    def dq_forward(self, dofs, weights):
        dofs, weights = _f32(dofs, "dofs"), _f32(weights, "skinning_weights")
        B = dofs.shape[0]
        o = self._outs(B, dofs.device, 8)
        P = _lib.ptr
        _lib.call("hc_dq_skinning_forward", self._h, _stream(), B, P(dofs), P(weights), *(P(t) for t in o))
        return o

    def dq_backward(self, gv, vpos, gpos, gaxis, dq, weights):
        args = [_f32(t, n) for t, n in ((gv, "grad"), (vpos, "positions"), (gpos, "joint_pos"), (gaxis, "joint_axis"),
                                        (dq, "dual_quaternions"), (weights, "weights"))]
        B = args[0].shape[0]
        gd = torch.empty((B, self.D), device=args[0].device)
        gw = torch.empty((B, self.N, self.K), device=args[0].device)
        P = _lib.ptr
        _lib.call("hc_dq_skinning_backward", self._h, _stream(), B, *(P(t) for t in args), P(gd), P(gw))
        return gd, gw

    def pose2eg(self, dofs, node_vertex, weights):
        """Pose2EmbeddedGraphCpu on the device (Pose2EmbeddedGraphCPUOp.cpp:129-300).

        dofs [B,D]; node_vertex [M] int32 (base vertex of each graph node);
        weights [N,K] (the character's skin weights).  Returns
        (nodes_skinned_translation [B,M,3], nodes_skinned_rotation [B,M,3] Z-Y-X
        Euler, dual_quaternions [B,S,8])."""
        dofs, weights = _f32(dofs, "dofs"), _f32(weights, "skinning_weights")
        nv = node_vertex.to(torch.int32).contiguous() if torch.is_tensor(node_vertex) else \
            torch.as_tensor(node_vertex, dtype=torch.int32, device=dofs.device)
        if weights.shape != (self.N, self.K):
            raise ValueError(f"skin weights must be [{self.N},{self.K}], got {tuple(weights.shape)}")
        if nv.numel() and (int(nv.min()) < 0 or int(nv.max()) >= self.N):
            raise ValueError("node_vertex index out of range")
        B, M = dofs.shape[0], nv.numel()
        t = torch.empty((B, M, 3), device=dofs.device)
        a = torch.empty((B, M, 3), device=dofs.device)
        dq = torch.empty((B, self.S, 8), device=dofs.device)
        P = _lib.ptr
        _lib.call("hc_pose2eg_forward", self._h, _stream(), B, P(dofs), M, P(nv), P(weights), P(t), P(a), P(dq))
        return t, a, dq

    def pose2eg_backward(self, dofs, node_vertex, weights, grad_translation, grad_rotation):
        """Adjoint of ``pose2eg``: d loss / d dofs [B,D] from the gradients of
        the node translations / Euler rotations [B,M,3] (the reference op
        has no gradient; this one is exact)."""
        dofs, weights = _f32(dofs, "dofs"), _f32(weights, "skinning_weights")
        gt, ga = _f32(grad_translation, "grad_translation"), _f32(grad_rotation, "grad_rotation")
        nv = node_vertex.to(torch.int32).contiguous() if torch.is_tensor(node_vertex) else \
            torch.as_tensor(node_vertex, dtype=torch.int32, device=dofs.device)
        B, M = dofs.shape[0], nv.numel()
        out = torch.empty((B, self.D), device=dofs.device)
        P = _lib.ptr
        _lib.call("hc_pose2eg_backward", self._h, _stream(), B, P(dofs), M, P(nv), P(weights), P(gt), P(ga), P(out))
        return out

    def lbs_forward(self, dofs, weights, disp):
        dofs, weights, disp = _f32(dofs, "dofs"), _f32(weights, "skinning_weights"), _f32(disp, "displacement")
        B = dofs.shape[0]
        o = self._outs(B, dofs.device, 12)
        P = _lib.ptr
        _lib.call("hc_lb_skinning_forward", self._h, _stream(), B, P(dofs), P(weights), P(disp), *(P(t) for t in o))
        return o

    def lbs_backward(self, gv, vpos, gpos, gaxis, xf, weights, disp=None):
        args = [_f32(t, n) for t, n in ((gv, "grad"), (vpos, "positions"), (gpos, "joint_pos"), (gaxis, "joint_axis"),
                                        (xf, "transformation"), (weights, "weights"))]
        B = args[0].shape[0]
        dev = args[0].device
        gd = torch.empty((B, self.D), device=dev)
        gw = torch.empty((B, self.N, self.K), device=dev)
        gdisp = torch.empty((B, self.N, 3), device=dev)
        P = _lib.ptr
        _lib.call("hc_lb_skinning_backward", self._h, _stream(), B, *(P(t) for t in args),
                  P(_f32(disp, "displacement")) if disp is not None else None, P(gd), P(gw), P(gdisp))
        return gd, gw, gdisp


class _DQFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eng: SkinningEngine, dofs, weights):
        v, n, gp, ga, dq, w = eng.dq_forward(dofs, weights)
        ctx.eng = eng
        ctx.save_for_backward(v, gp, ga, dq, w)
        ctx.mark_non_differentiable(gp, ga, dq, w)
        return v, n, gp, ga, dq, w

    @staticmethod
    def backward(ctx, gv, gn, ggp, gga, gdq, gw):
        v, gp, ga, dq, w = ctx.saved_tensors
        if gv is None:
            gv = torch.zeros_like(v)
        gd, gwt = ctx.eng.dq_backward(gv, v, gp, ga, dq, w)
        return None, gd, gwt


class _LBSFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eng: SkinningEngine, dofs, weights, disp):
        v, n, gp, ga, xf, w = eng.lbs_forward(dofs, weights, disp)
        ctx.eng = eng
        ctx.save_for_backward(v, gp, ga, xf, w, disp)
        ctx.mark_non_differentiable(gp, ga, xf, w)
        return v, n, gp, ga, xf, w

    @staticmethod
    def backward(ctx, gv, gn, ggp, gga, gxf, gw):
        v, gp, ga, xf, w, disp = ctx.saved_tensors
        if gv is None:
            gv = torch.zeros_like(v)
        gd, gwt, gdisp = ctx.eng.lbs_backward(gv, v, gp, ga, xf, w, disp)
        return None, gd, gwt, gdisp


def dq_skinning_gpu(engine: SkinningEngine, dofs, skinning_weights):
    """``DqSkinningGpu``: (skinned_vertex_positions, skinned_vertex_normals, global_joint_position,
    global_joint_axis, dual_quaternions, output_skinning_weights), differentiable in dofs and weights."""
    return _DQFn.apply(engine, dofs, skinning_weights)


def lb_skinning_gpu(engine: SkinningEngine, dofs, skinning_weights, displacement):
    """``LbSkinningGpu``: (skinned positions, normals, joint positions, joint axes, transformation,
    output weights), differentiable in dofs, weights and displacement."""
    return _LBSFn.apply(engine, dofs, skinning_weights, displacement)
