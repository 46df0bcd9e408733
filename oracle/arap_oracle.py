"""Test oracle, never imported by the product: FP64 restatement of the
embedded-graph ARAP regulariser on the CPU (numpy), used by tests/ as the
checker.

Follows CustomTensorFlowCPPOperators/src/CustomGPUOperators/
EmbeddedGraphARAPOperator/EmbeddedGraphArapGPUOp.cu:10-97 (forward) and
EmbeddedGraphArapGPUOpGrad.cu:9-96 (adjoint), with the rotation
R = Rz(c) Ry(b) Rx(a) of CudaUtils/EmbeddedGraphRotationHelper.h:53-191.
Pinned to the reference kernels by tests/golden/arap.npz (made by
tests/golden/make_golden.py from oracle/_ref)."""
import numpy as np


def euler_rot(a):
    """R(a) [..., 3, 3] (EmbeddedGraphRotationHelper.h:53-77)."""
    a = np.asarray(a, np.float64)
    ca, cb, cg = np.cos(a[..., 0]), np.cos(a[..., 1]), np.cos(a[..., 2])
    sa, sb, sg = np.sin(a[..., 0]), np.sin(a[..., 1]), np.sin(a[..., 2])
    R = np.empty(a.shape[:-1] + (3, 3))
    R[..., 0, 0] = cb * cg
    R[..., 0, 1] = sa * sb * cg - ca * sg
    R[..., 0, 2] = ca * sb * cg + sa * sg
    R[..., 1, 0] = cb * sg
    R[..., 1, 1] = sa * sb * sg + ca * cg
    R[..., 1, 2] = ca * sb * sg - sa * cg
    R[..., 2, 0] = -sb
    R[..., 2, 1] = sa * cb
    R[..., 2, 2] = ca * cb
    return R


def euler_rot_d(a):
    """dR/da, dR/db, dR/dc [3, ..., 3, 3] (EmbeddedGraphRotationHelper.h:109-191), by
    differentiating the product of the three axis rotations."""
    a = np.asarray(a, np.float64)
    ca, cb, cg = np.cos(a[..., 0]), np.cos(a[..., 1]), np.cos(a[..., 2])
    sa, sb, sg = np.sin(a[..., 0]), np.sin(a[..., 1]), np.sin(a[..., 2])
    z, o = np.zeros_like(ca), np.ones_like(ca)

    def m(*rows):
        return np.stack([np.stack(r, -1) for r in rows], -2)
    Rx, Ry, Rz = m((o, z, z), (z, ca, -sa), (z, sa, ca)), m((cb, z, sb), (z, o, z), (-sb, z, cb)), \
        m((cg, -sg, z), (sg, cg, z), (z, z, o))
    dRx, dRy, dRz = m((z, z, z), (z, -sa, -ca), (z, ca, -sa)), m((-sb, z, cb), (z, z, z), (-cb, z, -sb)), \
        m((-sg, -cg, z), (cg, -sg, z), (z, z, z))
    return Rz @ Ry @ dRx, Rz @ dRy @ Rx, dRz @ Ry @ Rx


def arap_forward(base, node_vertex, off, size, idx, rigid, maxc, T, A):
    """(nodes_arap_loss [B,M,maxc,3], connection_weights [B,M,maxc], rotation [B,M,3])
    (EmbeddedGraphArapGPUOp.cu:10-92)."""
    T, A = np.asarray(T, np.float64), np.asarray(A, np.float64)
    B, M = T.shape[:2]
    g = np.asarray(base, np.float64)[np.asarray(node_vertex)]
    R = euler_rot(A)
    loss = np.zeros((B, M, maxc, 3))
    w = np.zeros((B, M, maxc))
    for j in range(M):
        for s in range(size[j]):
            k = idx[off[j] + s]
            loss[:, j, s] = np.einsum("bij,j->bi", R[:, j], g[k] - g[j]) + g[j] + T[:, j] - (g[k] + T[:, k])
            w[:, j, s] = (rigid[j] + rigid[k]) / 2.0
    return loss, w, A.copy()


def arap_backward(base, node_vertex, off, size, idx, maxc, gloss, A):
    """(nodes_t_grad, nodes_r_grad) [B,M,3] (EmbeddedGraphArapGPUOpGrad.cu:9-96):
    dT_j = sum_s (gbar_js - gbar_k s'), s' the last slot of j in k's list."""
    gloss, A = np.asarray(gloss, np.float64), np.asarray(A, np.float64)
    B, M = A.shape[:2]
    g = np.asarray(base, np.float64)[np.asarray(node_vertex)]
    dR = euler_rot_d(A)
    gT = np.zeros((B, M, 3))
    gA = np.zeros((B, M, 3))
    for j in range(M):
        for s in range(size[j]):
            k = idx[off[j] + s]
            d = g[k] - g[j]
            r = gloss[:, j, s]
            for c in range(3):
                gA[:, j, c] += np.einsum("bi,bi->b", np.einsum("bij,j->bi", dR[c][:, j], d), r)
            rk = np.zeros((B, 3))
            for q in range(size[k]):
                if idx[off[k] + q] == j:
                    rk = gloss[:, k, q]
            gT[:, j] += r - rk
    return gT, gA
