"""The added bilinear texture mode (``texturedBilinear``, no reference
counterpart: the reference's textured mode samples the nearest texel) against
a torch FP64 restatement differentiated by autograd: forward colours,
texture gradient and vertex-position gradient (through the barycentrics of
the ray hit, visibility fixed to the rendered face buffer).  The target image
is zero so that the renderer's data-term gradient vanishes."""
import numpy as np
import pytest
import torch

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.renderer import RendererEngine, renderer_backward

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def nrel(a, b):
    a, b = a.double().cpu(), b.double().cpu()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


def torch_bilinear_render(verts, tex, faces, texcoords, extr, intr, face_buf, W, H):
    """FP64 colours of the covered pixels and their (view, y, x) index."""
    B, C = face_buf.shape[:2]
    out, idx = [], []
    f_all = torch.as_tensor(faces, dtype=torch.long, device=DEV)
    tc = torch.as_tensor(texcoords, dtype=torch.float64, device=DEV).reshape(-1, 3, 2)
    TH, TW = tex.shape[1], tex.shape[2]
    for b in range(B):
        for c in range(C):
            E = torch.as_tensor(extr[b, 12 * c:12 * c + 12], dtype=torch.float64, device=DEV).reshape(3, 4)
            K = torch.as_tensor(intr[b, 9 * c:9 * c + 9], dtype=torch.float64, device=DEV).reshape(3, 3)
            R, t = E[:, :3], E[:, 3]
            o = -R.T @ t
            yy, xx = torch.nonzero(face_buf[b, c] >= 0, as_tuple=True)
            f = face_buf[b, c][yy, xx].long()
            pix = torch.stack([xx.double() + 0.5, yy.double() + 0.5, torch.ones_like(xx, dtype=torch.float64)], 1)
            d = (torch.linalg.inv(K) @ pix.T).T @ R  # R^T applied to each row
            d = d / d.norm(dim=1, keepdim=True)
            tri = f_all[f]
            v0, v1, v2 = verts[b][tri[:, 0]], verts[b][tri[:, 1]], verts[b][tri[:, 2]]
            N = torch.cross(v1 - v0, v2 - v0, dim=1)
            tt = ((v0 - o) * N).sum(1) / (d * N).sum(1)
            P = o + tt[:, None] * d
            den = (N * N).sum(1)
            a = (N * torch.cross(v2 - v1, P - v1, dim=1)).sum(1) / den
            bb = (N * torch.cross(v0 - v2, P - v2, dim=1)).sum(1) / den
            cc = 1 - a - bb
            t3 = tc[f]
            u = t3[:, 0, 0] * a + t3[:, 1, 0] * bb + t3[:, 2, 0] * cc
            v = (1 - t3[:, 0, 1]) * a + (1 - t3[:, 1, 1]) * bb + (1 - t3[:, 2, 1]) * cc
            sx, sy = u * TW - 0.5, v * TH - 0.5
            x0, y0 = torch.floor(sx).detach(), torch.floor(sy).detach()
            fx, fy = sx - x0, sy - y0
            xa, xb = x0.long().clamp(0, TW - 1), (x0.long() + 1).clamp(0, TW - 1)
            ya, yb = y0.long().clamp(0, TH - 1), (y0.long() + 1).clamp(0, TH - 1)
            T = tex[b]
            col = (T[ya, xa] * ((1 - fx) * (1 - fy))[:, None] + T[ya, xb] * (fx * (1 - fy))[:, None] +
                   T[yb, xa] * ((1 - fx) * fy)[:, None] + T[yb, xb] * (fx * fy)[:, None])
            out.append(col)
            idx.append((b, c, yy, xx))
    return out, idx


def test_bilinear_mode_matches_torch_fp64_autograd():
    sc = S.render_scene(3, batch=1, views=2, width=64, height=48, seed=23, texture_size=32)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    verts, colors, tex, sh = t(sc["verts"]), t(sc["colors"]), t(sc["texture"]), t(sc["sh"])
    extr, intr = t(sc["extr"]), t(sc["intr"])
    eng = RendererEngine(sc["faces"], sc["texcoords"], sc["N"], 2, 64, 48, "texturedBilinear", "shadeless", 2, 2)
    bary, face, render, vn, _ = eng.forward(verts, colors, tex, sh, extr, intr)
    G = torch.randn(render.shape, device=DEV, generator=torch.Generator(DEV).manual_seed(4))
    target = torch.zeros_like(render)
    gpos, _, gtex, _ = renderer_backward(eng, G, verts, colors, tex, sh, target, vn, bary, face, extr, intr)
    torch.cuda.synchronize()
    assert int((face >= 0).sum()) > 500
    v64 = verts.double().requires_grad_(True)
    t64 = tex.double().requires_grad_(True)
    cols, idx = torch_bilinear_render(v64, t64, sc["faces"], sc["texcoords"], sc["extr"], sc["intr"], face, 64, 48)
    L = 0
    for col, (b, c, yy, xx) in zip(cols, idx):
        assert float((render[b, c, yy, xx].double() - col).abs().max()) < 1e-4
        L = L + (G[b, c, yy, xx].double() * col).sum()
    L.backward()
    assert nrel(gtex, t64.grad) < 5e-5  # FP32 atomics summing many pixels per texel
    assert nrel(gpos, v64.grad) < 1e-4, nrel(gpos, v64.grad)
