"""UV-space normal / position / face maps (compute_normal_map) against the
reference renderer object (its own host texel table + kernels) and the FP64
texel-table restatement."""
import numpy as np
import pytest
import torch

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.renderer import RendererEngine
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference kernels (oracle/_ref) not built")
RES, TEX = 96, 64


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.fixture(scope="module")
def scene():
    return S.render_scene(3, batch=2, views=2, width=RES, height=RES, seed=21, texture_size=TEX)


@needs_ref
@pytest.mark.parametrize("mode", ["normal", "position", "face"])
def test_uv_map_matches_reference(scene, mode):
    sc = scene
    eng = RendererEngine(sc["faces"], sc["texcoords"], sc["N"], 2, RES, RES, "vertexColor", "shadeless", 2, 2, mode)
    tex = _t(sc["texture"])
    out = eng.forward(_t(sc["verts"]), _t(sc["colors"]), tex, _t(sc["sh"]), _t(sc["extr"]), _t(sc["intr"]))
    bary, face, render, vnormal, nmap = out[:5]
    ref = O.RefUV(sc["faces"], sc["texcoords"], sc["N"], 2, RES, RES, mode).forward(
        2, _t(sc["verts"]), _t(sc["extr"]), _t(sc["intr"]), TEX, TEX)
    torch.cuda.synchronize()
    assert torch.equal(face, ref["face"]) and bool((face == -1).all())
    assert torch.equal(bary, ref["bary"]) and torch.equal(render, ref["render"])
    assert torch.equal(vnormal, ref["vnormal"])
    assert float(nmap.abs().sum()) > 0
    assert torch.equal(nmap, ref["normal_map"]), int((nmap != ref["normal_map"]).any(-1).sum())


def test_texel_table_matches_fp64_oracle(scene):
    sc = scene
    eng = RendererEngine(sc["faces"], sc["texcoords"], sc["N"], 2, RES, RES, "vertexColor", "shadeless", 2, 2, "face")
    tex = _t(sc["texture"])
    nmap = eng.forward(_t(sc["verts"]), _t(sc["colors"]), tex, _t(sc["sh"]), _t(sc["extr"]), _t(sc["intr"]))[4]
    ours = nmap[0, :, :, 0].cpu().numpy()
    ora = O.texel_table(sc["texcoords"], TEX, TEX)
    # texels whose centre lies on a UV edge can go to either neighbour
    assert (ours != ora[..., 0]).mean() < 0.02
    assert (ora[..., 0] > 0).mean() > 0.5
