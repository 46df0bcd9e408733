"""FP64 restatement of forward kinematics and DQ / LBS skinning -- TEST ORACLE.

Follows Skeletool/Character/joint.cpp:36-116,144-168 (joint chain: parent *
translate(offset * scale) * rotation about the local axis / translation
along it), dof.cpp:9-17 (dof -> joint parameters), DQSkinningGPUOp.cpp:
257-347 (skinning transform joint * scale * inverse(rest), DualQuaternion.h:
58-69), DQSkinningGPUOp.cu:56-120 (sign-aligned blend, normalisation),
LBSkinningGPUOp.cu:49-96 (blended rotation / translation) and the gradient
kernels DQSkinningGPUOpGrad.cu:145-206 / LBSkinningGPUOpGrad.cu:93-154 (dof
gradient sum over (vertex, bone, joint-on-chain) of w (axis x (v - c)) . g).
Eigen is not available, so the reference's host kinematics cannot be run
here; this restatement is cross-checked internally (zero pose -> identity,
matrix chain vs dual-quaternion transform, finite differences).
Only tests import this module.
"""
from __future__ import annotations

import numpy as np


def axis_angle(a, th):
    a = np.asarray(a, np.float64)
    c, s = np.cos(th), np.sin(th)
    x, y, z = a
    C = 1 - c
    return np.array([[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                     [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                     [z * x * C - y * s, z * y * C + x * s, c + z * z * C]])


def fk(ch, dofs, unit_scale=False):
    """Joint transforms (R [B,J,3,3], t [B,J,3]), global positions and axes [B,J,3].

    ``unit_scale``: every joint scale taken as 1, as in the bind pose
    (Skeletool/Character/skeleton.cpp:2840-2853)."""
    dofs = np.asarray(dofs, np.float64)
    B = dofs.shape[0]
    J = ch.n_joints
    js = np.ones(J) if ch.joint_scale is None or unit_scale else np.asarray(ch.joint_scale, np.float64)
    R = np.zeros((B, J, 3, 3))
    t = np.zeros((B, J, 3))
    gaxis = np.zeros((B, J, 3))
    for b in range(B):
        P = np.zeros(J)
        for d in range(ch.n_dofs):
            for e in range(ch.dof_offsets[d], ch.dof_offsets[d + 1]):
                P[ch.dof_joint[e]] += ch.dof_weight[e] * dofs[b, d]
        for j in range(J):
            ax = np.asarray(ch.axis[j], np.float64)
            lt = np.asarray(ch.offset[j], np.float64) * js[j]
            if ch.joint_type[j] == 0:
                lr = axis_angle(ax, P[j])
            else:
                lr = np.eye(3)
                lt = lt + ax * P[j]
            p = ch.parent[j]
            if p >= 0:
                R[b, j] = R[b, p] @ lr
                t[b, j] = R[b, p] @ lt + t[b, p]
            else:
                R[b, j] = lr
                t[b, j] = lt
            gaxis[b, j] = R[b, j] @ ax
    return R, t, t.copy(), gaxis


def skin_transforms(ch, dofs):
    """Per skinning joint: joint * scale * inverse(bind joint) as (R [B,S,3,3], t [B,S,3]).

    The bind transforms are taken at zero dofs with unit joint scales
    (skinnedcharacter.cpp:178-183 after skeleton.cpp:2840-2853)."""
    R, t, _, _ = fk(ch, dofs)
    R0, t0, _, _ = fk(ch, np.zeros((1, ch.n_dofs)), unit_scale=True)
    S = ch.n_skin
    ss = np.ones(S) if ch.skin_scale is None else np.asarray(ch.skin_scale, np.float64)
    B = R.shape[0]
    Rs = np.zeros((B, S, 3, 3))
    ts = np.zeros((B, S, 3))
    for s in range(S):
        j = ch.skin_joint[s]
        Ri = R0[0, j].T
        ti = -Ri @ t0[0, j]
        for b in range(B):
            Rs[b, s] = R[b, j] @ Ri  # the uniform scale cancels in the rotation part
            ts[b, s] = R[b, j] @ (ss[s] * ti) + t[b, j]
    return Rs, ts


def mat_to_quat(R):
    """(x, y, z, w) of a rotation matrix (Shepperd's method)."""
    tr = np.trace(R)
    q = np.zeros(4)
    if tr > 0:
        s = np.sqrt(tr + 1.0)
        q[3] = 0.5 * s
        s = 0.5 / s
        q[0] = (R[2, 1] - R[1, 2]) * s
        q[1] = (R[0, 2] - R[2, 0]) * s
        q[2] = (R[1, 0] - R[0, 1]) * s
    else:
        i = int(np.argmax(np.diag(R)))
        j, k = (i + 1) % 3, (i + 2) % 3
        s = np.sqrt(R[i, i] - R[j, j] - R[k, k] + 1.0)
        q[i] = 0.5 * s
        s = 0.5 / s
        q[3] = (R[k, j] - R[j, k]) * s
        q[j] = (R[j, i] + R[i, j]) * s
        q[k] = (R[k, i] + R[i, k]) * s
    return q / np.linalg.norm(q)


def dual_quaternions(ch, dofs):
    Rs, ts = skin_transforms(ch, dofs)
    B, S = Rs.shape[:2]
    dq = np.zeros((B, S, 8))
    for b in range(B):
        for s in range(S):
            q = mat_to_quat(Rs[b, s])
            t = ts[b, s]
            dq[b, s, :4] = q
            dq[b, s, 7] = -0.5 * (t @ q[:3])
            dq[b, s, 4] = 0.5 * (t[0] * q[3] + t[1] * q[2] - t[2] * q[1])
            dq[b, s, 5] = 0.5 * (-t[0] * q[2] + t[1] * q[3] + t[2] * q[0])
            dq[b, s, 6] = 0.5 * (t[0] * q[1] - t[1] * q[0] + t[2] * q[3])
    return dq


def quat_rot(q):
    x, y, z, w = q
    return np.array([[1 - 2 * y * y - 2 * z * z, 2 * y * x - 2 * z * w, 2 * z * x + 2 * y * w],
                     [2 * y * x + 2 * z * w, 1 - 2 * x * x - 2 * z * z, 2 * z * y - 2 * x * w],
                     [2 * z * x - 2 * y * w, 2 * z * y + 2 * x * w, 1 - 2 * x * x - 2 * y * y]])


def dq_trans(r, t):
    return 2 * np.array([-t[3] * r[0] + t[0] * r[3] - t[1] * r[2] + t[2] * r[1],
                         -t[3] * r[1] + t[0] * r[2] + t[1] * r[3] - t[2] * r[0],
                         -t[3] * r[2] - t[0] * r[1] + t[1] * r[0] + t[2] * r[3]])


def dq_skin(ch, dq, weights):
    """Skinned positions / normals [B,N,3] from dual quaternions [B,S,8] and weights [B,N,K]."""
    dq = np.asarray(dq, np.float64)
    w = np.asarray(weights, np.float64)
    B = dq.shape[0]
    N, K = ch.skin_index.shape
    out_v = np.zeros((B, N, 3))
    out_n = np.zeros((B, N, 3))
    for b in range(B):
        for v in range(N):
            br = np.zeros(4)
            bt = np.zeros(4)
            first = dq[b, ch.skin_index[v, 0], :4]
            for k in range(K):
                q = dq[b, ch.skin_index[v, k]]
                sign = -1.0 if (k != 0 and first @ q[:4] < 0) else 1.0
                br += q[:4] * w[b, v, k] * sign
                bt += q[4:] * w[b, v, k] * sign
            n = np.linalg.norm(br)
            if n > 1e-6:
                br /= n
                bt /= n
            Rm = quat_rot(br)
            out_v[b, v] = Rm @ ch.base_vertices[v] + dq_trans(br, bt)
            rn = Rm @ ch.base_normals[v]
            out_n[b, v] = rn / np.linalg.norm(rn)
    return out_v, out_n


def pose2eg(ch, dofs, node_vertex, weights):
    """Node-level skinning of the embedded graph in FP64
    (Pose2EmbeddedGraphCPUOp.cpp:129-300): blend the dual quaternions of each
    node's base vertex with the skin weights [N,K] (sign-aligned to the first,
    normalised when the norm exceeds 1e-6), return the blended translation and
    the Z-Y-X Euler angles of the blended rotation (singular branch for
    sy < 1e-6), [B,M,3] each, plus the joints' dual quaternions [B,S,8]."""
    dq = dual_quaternions(ch, dofs)
    w = np.asarray(weights, np.float64)
    nv = np.asarray(node_vertex, np.int64)
    idx = ch.skin_index[nv]                      # [M,K]
    q = dq[:, idx]                               # [B,M,K,8]
    wk = w[nv][None, :, :, None]                 # [1,M,K,1]
    first = q[:, :, :1, :4]
    sign = np.where(np.sum(first * q[..., :4], -1, keepdims=True) < 0, -1.0, 1.0)
    sign[:, :, 0] = 1.0
    blend = np.sum(q * wk * sign, axis=2)        # [B,M,8]
    ln = np.linalg.norm(blend[..., :4], axis=-1, keepdims=True)
    blend = np.where(ln > 1e-6, blend / np.where(ln > 1e-6, ln, 1.0), blend)
    r, t = blend[..., :4], blend[..., 4:]
    x, y, z, ww = r[..., 0], r[..., 1], r[..., 2], r[..., 3]
    tx, ty, tz, tw = t[..., 0], t[..., 1], t[..., 2], t[..., 3]
    out_t = 2 * np.stack([-tw * x + tx * ww - ty * z + tz * y,
                          -tw * y + tx * z + ty * ww - tz * x,
                          -tw * z - tx * y + ty * x + tz * ww], -1)
    R00 = 1 - 2 * y * y - 2 * z * z
    R10 = 2 * y * x + 2 * z * ww
    R20 = 2 * z * x - 2 * y * ww
    R21 = 2 * z * y + 2 * x * ww
    R22 = 1 - 2 * x * x - 2 * y * y
    R11 = 1 - 2 * x * x - 2 * z * z
    R12 = 2 * z * y - 2 * x * ww
    sy = np.hypot(R00, R10)
    sing = sy < 1e-6
    ax = np.where(sing, np.arctan2(-R12, R11), np.arctan2(R21, R22))
    ay = np.arctan2(-R20, sy)
    az = np.where(sing, 0.0, np.arctan2(R10, R00))
    return out_t, np.stack([ax, ay, az], -1), dq


def lbs_skin(ch, Rs, ts, weights, disp):
    w = np.asarray(weights, np.float64)
    disp = np.asarray(disp, np.float64)
    idx = ch.skin_index
    Rb = np.einsum("bvk,bvkij->bvij", w, Rs[:, idx])
    tb = np.einsum("bvk,bvki->bvi", w, ts[:, idx])
    p = ch.base_vertices[None].astype(np.float64) + disp
    return np.einsum("bvij,bvj->bvi", Rb, p) + tb, np.einsum("bvij,vj->bvi", Rb, ch.base_normals.astype(np.float64))


def dof_grad_reference(ch, vpos, gv, weights, gpos, gaxis):
    """The reference's linearised dof gradient (DQSkinningGPUOpGrad.cu:145-206)."""
    vpos = np.asarray(vpos, np.float64)
    gv = np.asarray(gv, np.float64)
    w = np.asarray(weights, np.float64)
    B = vpos.shape[0]
    D = ch.n_dofs
    out = np.zeros((B, D))
    N, K = ch.skin_index.shape
    for b in range(B):
        for d in range(D):
            joints = set(ch.dof_joint[ch.dof_offsets[d]:ch.dof_offsets[d + 1]].tolist())
            acc = 0.0
            for v in range(N):
                for k in range(K):
                    pr = ch.skin_joint[ch.skin_index[v, k]]
                    while pr >= 0:
                        if pr in joints:
                            ax = gaxis[b, pr]
                            r = np.cross(ax, vpos[b, v] - gpos[b, pr]) if ch.joint_type[pr] == 0 else ax
                            acc += w[b, v, k] * (r @ gv[b, v])
                        pr = ch.parent[pr]
            out[b, d] = acc
    return out
