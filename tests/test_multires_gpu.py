"""Views of different resolutions in one launch (config 3's batching: per-view
resolutions from {512x512, 768x1024, 1024x1024, 1536x1024}).  Each camera's
slice of the mixed-size call must be bit-identical to a single-camera call of
that size (the uniform path is checked against the reference kernels), and
the adjoint must equal the sum of the single-camera adjoints."""
import numpy as np
import pytest
import torch

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.renderer import RendererEngine, renderer_backward

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
SIZES = [(512, 512), (768, 1024), (1024, 1024), (1536, 1024)]  # (W, H)


def nrel(a, b):
    a, b = a.double(), b.double()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


def cameras(B):
    ex, it = [], []
    for c, (w, h) in enumerate(SIZES):
        e, k = S.camera_ring(len(SIZES), 3000.0, 600.0 * min(w, h) / 512, w, h)
        ex.append(e[12 * c:12 * c + 12])
        it.append(k[9 * c:9 * c + 9])
    return np.tile(np.concatenate(ex)[None], (B, 1)), np.tile(np.concatenate(it)[None], (B, 1))


@pytest.mark.parametrize("tile", [8, 16, 32])
def test_mixed_resolution_views_match_single_camera_calls(tile):
    B = 2
    sc = S.render_scene(4, batch=B, views=len(SIZES), width=64, height=64, seed=29, texture_size=32)
    extr, intr = cameras(B)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(DEV)  # noqa: E731
    verts, colors, tex = t(sc["verts"]), t(sc["colors"]), t(sc["texture"])
    sh = t(sc["sh"])
    W = [w for w, _ in SIZES]
    H = [h for _, h in SIZES]
    eng = RendererEngine(sc["faces"], sc["texcoords"], sc["N"], len(SIZES), W, H, "vertexColor", "shaded", 2, 2)
    eng.set_tuning(tile, 256)
    assert eng.multires and eng.P_frame == sum(w * h for w, h in SIZES)
    bary, face, render, vn, _ = eng.forward(verts, colors, tex, sh, t(extr), t(intr))
    target = torch.rand(render.shape, device=DEV, generator=torch.Generator(DEV).manual_seed(1))
    G = torch.randn(render.shape, device=DEV, generator=torch.Generator(DEV).manual_seed(2))
    gpos, gcol, _, gsh = renderer_backward(eng, G, verts, colors, tex, sh, target, vn, bary, face, t(extr), t(intr))
    torch.cuda.synchronize()
    parts = {k: eng.split_views(v) for k, v in (("bary", bary), ("face", face), ("render", render),
                                              ("target", target), ("G", G))}
    sum_pos = torch.zeros_like(gpos)
    sum_col = torch.zeros_like(gcol)
    for c, (w, h) in enumerate(SIZES):
        one = RendererEngine(sc["faces"], sc["texcoords"], sc["N"], 1, w, h, "vertexColor", "shaded", 2, 2)
        one.set_tuning(tile, 256)
        ex1, in1 = t(extr[:, 12 * c:12 * c + 12]), t(intr[:, 9 * c:9 * c + 9])
        b1, f1, r1, vn1, _ = one.forward(verts, colors, tex, sh[:, c:c + 1], ex1, in1)
        assert torch.equal(parts["face"][c], f1[:, 0]), c
        assert torch.equal(parts["bary"][c], b1[:, 0]) and torch.equal(parts["render"][c], r1[:, 0]), c
        assert torch.equal(vn[:, c], vn1[:, 0])
        tg = parts["target"][c].unsqueeze(1).contiguous()
        g1 = parts["G"][c].unsqueeze(1).contiguous()
        p1, c1, _, s1 = renderer_backward(one, g1, verts, colors, tex, sh[:, c:c + 1], tg, vn1, b1, f1, ex1, in1)
        sum_pos += p1
        sum_col += c1
        assert nrel(gsh[:, c], s1[:, 0]) < 1e-5  # float sums in a different order
    torch.cuda.synchronize()
    assert nrel(gpos, sum_pos) < 1e-5 and nrel(gcol, sum_col) < 1e-5
