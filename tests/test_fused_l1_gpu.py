"""The image L1 fused into the raster (hc_renderer_forward_l1 /
hc_renderer_backward_l1) against the separate ops (hc_renderer_forward +
hc_image_l1_loss + hc_renderer_backward)."""
import numpy as np
import pytest
import torch

from deepcharacters_b200 import _lib
from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.chain import DeformRenderChain
from deepcharacters_b200.losses import image_l1_loss
from deepcharacters_b200.renderer import RendererEngine, _stream, renderer_backward

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def nrel(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


@pytest.mark.parametrize("albedo,shading,tile", [("vertexColor", "shadeless", 8), ("vertexColor", "shaded", 16),
                                                 ("textured", "shaded", 32)])
def test_fused_l1_matches_separate_ops(albedo, shading, tile):
    B, C, W, H = 2, 3, 96, 72
    sc = S.render_scene(3, batch=B, views=C, width=W, height=H, seed=13, texture_size=32)
    verts, colors, tex, sh = (_t(sc[k].astype(np.float32)) for k in ("verts", "colors", "texture", "sh"))
    ex, it = _t(sc["extr"].astype(np.float32)), _t(sc["intr"].astype(np.float32))
    # 8-bit targets, with exact ties (difference 0) on part of the pixels
    target = _t((np.random.default_rng(1).integers(0, 256, (B, C, H, W, 3)) / 255.0).astype(np.float32))
    mask = _t((np.random.default_rng(2).random((B, C, H, W)) < 0.8).astype(np.uint8))
    eng = RendererEngine(sc["faces"], sc["texcoords"], sc["N"], C, W, H, albedo, shading, 2, 2)
    eng.set_tuning(tile, 512)
    bary, face, render, vn, _ = eng.forward(verts, colors, tex, sh, ex, it)
    target[:, :, :H // 4] = render[:, :, :H // 4]  # zero differences are not counted
    loss, gimg = image_l1_loss(render, target, face, mask)
    ref = renderer_backward(eng, gimg, verts, colors, tex, sh, target, vn, bary, face, ex, it)
    torch.cuda.synchronize()

    o = {k: torch.empty_like(v) for k, v in (("bary", bary), ("face", face), ("render", render), ("vn", vn))}
    state = torch.zeros((2,), device=DEV, dtype=torch.float64)
    floss = torch.empty((1,), device=DEV)
    P = _lib.ptr
    TH, TW = int(tex.shape[1]), int(tex.shape[2])
    for _ in range(2):  # twice in a row: the state is rewritten, not accumulated
        _lib.call("hc_renderer_forward_l1", eng.handle, _stream(), B, P(verts), P(colors), P(tex), TH, TW, P(sh),
                  P(ex), P(it), P(o["bary"]), P(o["face"]), P(o["render"]), P(o["vn"]), P(target), P(mask),
                  P(state), P(floss))
    torch.cuda.synchronize()
    for k, v in (("bary", bary), ("face", face), ("render", render), ("vn", vn)):
        assert torch.equal(o[k], v), k
    assert nrel(floss, loss) < 1e-6
    grads = [torch.empty_like(ref[0]), torch.zeros_like(ref[1]), torch.zeros_like(ref[2]), torch.zeros_like(ref[3])]
    _lib.call("hc_renderer_backward_l1", eng.handle, _stream(), B, P(state), P(render), P(mask), P(verts),
              P(colors), P(tex), TH, TW, P(sh), P(target), P(vn), P(bary), P(face), P(ex), P(it), P(grads[0]),
              P(grads[1]), P(grads[2]) if albedo == "textured" else None, P(grads[3]))
    torch.cuda.synchronize()
    for name, a, b in zip(("pos", "col", "tex", "sh"), grads, ref):
        if float(b.abs().sum()) == 0.0:
            assert float(a.abs().sum()) == 0.0, name
        else:
            assert nrel(a, b) < 1e-5, name  # float atomics: summation order


def test_chain_fused_l1_matches_separate_ops():
    sc = S.chain_scene(3, 60, 4, 2, 3, 128, 96, seed=17)
    a = DeformRenderChain(sc, DEV, 2, 3, 128, 96, fused_l1=True)
    b = DeformRenderChain(sc, DEV, 2, 3, 128, 96, fused_l1=False)
    a.step()
    b.step()
    torch.cuda.synchronize()
    for k in ("face", "render", "bary", "isb"):
        assert torch.equal(a.buf[k], b.buf[k]), k
    assert nrel(a.loss, b.loss) < 1e-6
    for k in ("gT", "gA", "gcol", "gdofs"):
        assert nrel(a.buf[k], b.buf[k]) < 1e-5, k
