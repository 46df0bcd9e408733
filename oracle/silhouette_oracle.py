"""FP64 restatement of camera projection and the multi-view silhouette loss -- TEST ORACLE.

Follows CustomTensorFlowCPPOperators/src/CustomGPUOperators/CameraProjectionOperator/
CameraProjectionGPUOp.cu:12-86, CameraProjectionGPUOpGrad.cu:12-79 and
MultiViewSilhouetteLossOperator/MultiViewSilhouetteLossGPUOp.cu:11-240,
MultiViewSilhouetteLossGPUOpGrad.cu:11-59 (brute-force nearest boundary
vertex, as the reference does).  Only tests import this module.
"""
from __future__ import annotations

import numpy as np


def _cams(extr, intr, B, C):
    E = np.asarray(extr, np.float64).reshape(B, C, 3, 4)
    K = np.asarray(intr, np.float64).reshape(B, C, 3, 3)
    return E, K


def _proj(K, p):
    q = p @ K.T
    z = q[..., 2:3]
    z = np.where(z > 1e-7, z, 1e-5)
    return q[..., :2] / z


def project(points, vectors, extr, intr, is_point):
    P = np.asarray(points, np.float64)
    B, N = P.shape[:2]
    C = np.asarray(extr).reshape(B, -1).shape[1] // 12
    E, K = _cams(extr, intr, B, C)
    out = np.zeros((B, C, N, 2))
    for b in range(B):
        for c in range(C):
            cp = P[b] @ E[b, c, :, :3].T + E[b, c, :, 3]
            if is_point:
                out[b, c] = _proj(K[b, c], cp)
            else:
                np_ = cp + np.asarray(vectors, np.float64)[b] @ E[b, c, :, :3].T
                d = _proj(K[b, c], np_) - _proj(K[b, c], cp)
                out[b, c] = d / np.linalg.norm(d, axis=1, keepdims=True)
    return out


def project_grad(gimg, points, extr, intr):
    P = np.asarray(points, np.float64)
    B, N = P.shape[:2]
    C = gimg.shape[1]
    E, K = _cams(extr, intr, B, C)
    out = np.zeros((B, N, 3))
    for b in range(B):
        for c in range(C):
            cs = P[b] @ E[b, c, :, :3].T + E[b, c, :, 3]
            ax, ay, gm = K[b, c, 0, 0], K[b, c, 1, 1], K[b, c, 0, 1]
            z = cs[:, 2]
            dI = np.zeros((N, 2, 3))
            dI[:, 0, 0] = ax / z
            dI[:, 0, 1] = gm / z
            dI[:, 0, 2] = (-ax * cs[:, 0] - gm * cs[:, 1]) / z ** 2
            dI[:, 1, 1] = ay / z
            dI[:, 1, 2] = -ay * cs[:, 1] / z ** 2
            J = dI @ E[b, c, :, :3]
            out[b] += np.einsum("nij,ni->nj", J, gimg[b, c])
    return out


def _dec(v):
    v = v.astype(np.float64)
    return np.where(v >= 127, (v - 127) * 2, v)


def silhouette_forward(p2d, n2d, isb, dt, crops):
    """numpy FP64 forward; dt [B,C,U,V] stored with rows of U values."""
    p2d = np.asarray(p2d, np.float64)
    B, C, N = p2d.shape[:3]
    U, V = dt.shape[2], dt.shape[3]
    D = np.asarray(dt).reshape(B, C, V, U)
    res = np.zeros((B, C, N))
    dtg = np.zeros((B, C, N, 2))
    res1 = np.zeros((B, C, V, U, 2))
    closest = np.full((B, C, V, U), -1.0)
    for b in range(B):
        for c in range(C):
            cr = crops[b, c]
            sc = cr[2]
            Dv = D[b, c]
            for i in range(N):
                pu, pv = p2d[b, c, i]
                if not (pu - 2 > cr[3] and pu + 2 < cr[5] and pv - 2 > cr[4] and pv + 2 < cr[6]):
                    continue
                x = int((pu - cr[3]) / sc + cr[0])
                y = int((pv - cr[4]) / sc + cr[1])
                f = _dec(Dv[y - 1:y + 2, x - 1:x + 2])
                du = (-f[0, 0] + f[0, 2] - 2 * f[1, 0] + 2 * f[1, 2] - f[2, 0] + f[2, 2]) / 8
                dv = (-f[0, 0] - 2 * f[0, 1] - f[0, 2] + f[2, 0] + 2 * f[2, 1] + f[2, 2]) / 8
                inside = int(Dv[y, x]) <= 127
                dn = np.array([du, dv])
                dnu = dn.copy()
                if inside:
                    dn = -dn
                if not (dn @ n2d[b, c, i] >= 0) and inside:
                    dnu = -dnu
                w = float(bool(isb[b, c, i])) * float(du != 0 or dv != 0)
                res[b, c, i] = _dec(Dv[y, x]) * w / 255
                dtg[b, c, i] = dnu * w / 255
            bnd = np.nonzero(isb[b, c])[0]
            ys, xs = np.nonzero(Dv == 127)
            for y, x in zip(ys, xs):
                win = Dv[max(y - 2, 0):y + 3, max(x - 2, 0):x + 3]
                if (win == 127).sum() < 4:
                    continue
                ip = np.array([(x - cr[0]) * sc + cr[3], (y - cr[1]) * sc + cr[4]])
                if len(bnd) == 0:
                    continue
                d = np.linalg.norm(p2d[b, c, bnd] - ip, axis=1)
                k = int(np.argmin(d))
                if d[k] < 30 * sc:
                    v = bnd[k]
                    res1[b, c, y, x] = (p2d[b, c, v] - ip) / (30 * sc)
                    closest[b, c, y, x] = v
    return res, res1, dtg, closest


def silhouette_backward(g, g1, dtg, closest, crops):
    B, C, N = g.shape
    out = dtg * g[..., None]
    V, U = closest.shape[2:]
    for b in range(B):
        for c in range(C):
            sc = crops[b, c, 2]
            ys, xs = np.nonzero(closest[b, c] >= 0)
            for y, x in zip(ys, xs):
                out[b, c, int(closest[b, c, y, x])] += g1[b, c, y, x] / (30 * sc)
    return out


def mesh_boundary(faces, p2d, width, height):
    """ProjectedMeshBoundaryGpu in FP64 (Skeletool/Mesh/CUDABasedRasterization.cu:80-200):
    2-D coverage of every projected triangle (pixel centres with image-space
    barycentrics in [-0.001, 1.001] inside the clamped bounding box), then a
    vertex is a boundary vertex when its 3x3 window (around the truncated
    projection, fully inside the image) has an uncovered pixel.
    p2d [B,C,N,2] -> uint8 [B,C,N]."""
    p2d = np.asarray(p2d, np.float64)
    f = np.asarray(faces, np.int64).reshape(-1, 3)
    B, Cn, N = p2d.shape[:3]
    out = np.zeros((B, Cn, N), np.uint8)
    for b in range(B):
        for c in range(Cn):
            P = p2d[b, c]
            cover = np.zeros((height, width), bool)
            a, bb, cc = P[f[:, 0]], P[f[:, 1]], P[f[:, 2]]
            tri = np.stack([a, bb, cc], 1)
            x0 = np.maximum(tri[:, :, 0].min(1) - 0.5, 0).astype(np.int64)
            y0 = np.maximum(tri[:, :, 1].min(1) - 0.5, 0).astype(np.int64)
            x1 = np.minimum(tri[:, :, 0].max(1) + 0.5, width - 1).astype(np.int64)
            y1 = np.minimum(tri[:, :, 1].max(1) + 0.5, height - 1).astype(np.int64)
            d2 = (a[:, 1] - bb[:, 1]) * cc[:, 0] + (bb[:, 0] - a[:, 0]) * cc[:, 1] + a[:, 0] * bb[:, 1] - bb[:, 0] * a[:, 1]
            d1 = (a[:, 1] - cc[:, 1]) * bb[:, 0] + (cc[:, 0] - a[:, 0]) * bb[:, 1] + a[:, 0] * cc[:, 1] - cc[:, 0] * a[:, 1]
            for t in range(f.shape[0]):
                if x0[t] > x1[t] or y0[t] > y1[t]:
                    continue
                uu, vv = np.meshgrid(np.arange(x0[t], x1[t] + 1) + 0.5, np.arange(y0[t], y1[t] + 1) + 0.5)
                with np.errstate(divide="ignore", invalid="ignore"):
                    e2 = ((a[t, 1] - bb[t, 1]) * uu + (bb[t, 0] - a[t, 0]) * vv + a[t, 0] * bb[t, 1]
                          - bb[t, 0] * a[t, 1]) / d2[t]
                    e1 = ((a[t, 1] - cc[t, 1]) * uu + (cc[t, 0] - a[t, 0]) * vv + a[t, 0] * cc[t, 1]
                          - cc[t, 0] * a[t, 1]) / d1[t]
                e0 = 1.0 - e2 - e1
                ins = ((e0 >= -0.001) & (e1 >= -0.001) & (e2 >= -0.001) & (e0 <= 1.001) & (e1 <= 1.001)
                       & (e2 <= 1.001))
                cover[y0[t]:y1[t] + 1, x0[t]:x1[t] + 1] |= ins
            u = np.trunc(P[:, 0]).astype(np.int64)
            v = np.trunc(P[:, 1]).astype(np.int64)
            ok = (u - 1 >= 0) & (u + 1 < width) & (v - 1 >= 0) & (v + 1 < height)
            for i in np.nonzero(ok)[0]:
                out[b, c, i] = 0 if cover[v[i] - 1:v[i] + 2, u[i] - 1:u[i] + 2].all() else 1
    return out
