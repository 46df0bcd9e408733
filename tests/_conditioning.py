"""Pixels whose renderer gradient is well conditioned in FP32 (shared by the
adjoint tests that compare against the FP64 oracle).

At a grazing ray the barycentric derivative scales with 1/cos(ray, normal),
and so does its FP32 rounding, in the reference's formula and in the closed
form alike; textured gradients also contain discrete texel / tap choices
that flip under rounding.  The FP64 comparisons assert their 1e-5 bar on the
pixels this mask keeps and report the all-pixel number beside it.
"""
import numpy as np


def well_conditioned_mask(verts, faces, texcoords, tex_size, extr, intr, face, bary, albedo, min_cos=0.1,
                          margin=2e-3):
    """verts [B,N,3] (mm), faces [F,3], texcoords [F*6], extr [B,12C], intr [B,9C],
    face [B,C,H,W], bary [B,C,H,W,2] -> bool [B,C,H,W]: |cos(ray, normal)| >= min_cos
    and, for textured albedo, texel / tap choices not within `margin` of flipping."""
    B, C, H, W = face.shape
    tc = np.asarray(texcoords).reshape(-1, 3, 2)
    TH = TW = int(tex_size)
    m = np.zeros(face.shape, bool)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    for b in range(B):
        V = np.asarray(verts[b], np.float64)
        for c in range(C):
            E = np.eye(4)
            E[:3] = extr[b, 12 * c:12 * c + 12].reshape(3, 4)
            K = np.eye(4)
            K[:3, :3] = intr[b, 9 * c:9 * c + 9].reshape(3, 3)
            inv = np.linalg.inv(K @ E)
            o = np.linalg.inv(E)[:3, 3]
            pts = np.stack([(xx + 0.5) * 1000, (yy + 0.5) * 1000, np.full_like(xx, 1000.0), np.ones_like(xx)], -1)
            q = pts @ inv.T
            d = q[..., :3] - o
            d /= np.linalg.norm(d, axis=-1, keepdims=True)
            f = face[b, c]
            ok = f >= 0
            fi = np.where(ok, f, 0)
            v0, v1, v2 = V[faces[fi, 0]], V[faces[fi, 1]], V[faces[fi, 2]]
            n = np.cross(v1 - v0, v2 - v0)
            n /= np.maximum(np.linalg.norm(n, axis=-1, keepdims=True), 1e-300)
            good = ok & (np.abs((d * n).sum(-1)) >= min_cos)
            if albedo == "textured":
                a, bb = bary[b, c, ..., 0].astype(np.float64), bary[b, c, ..., 1].astype(np.float64)
                t = tc[fi]
                u = (t[..., 0, 0] * a + t[..., 1, 0] * bb + t[..., 2, 0] * (1 - a - bb)) * TW
                v = ((1 - t[..., 0, 1]) * a + (1 - t[..., 1, 1]) * bb + (1 - t[..., 2, 1]) * (1 - a - bb)) * TH
                fr = lambda x: np.minimum(np.mod(x, 1.0), 1 - np.mod(x, 1.0))  # noqa: E731
                good &= (fr(u - 0.5) > margin) & (fr(v - 0.5) > margin) & (fr(v * TW + u) > margin * TW)
            m[b, c] = good
    return m
