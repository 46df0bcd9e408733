"""The batched mixed-resolution chain: one call over frames x cameras whose
images differ in size, against the reference kernels run one camera size at
a time (the reference needs one op instance per resolution,
CudaRenderer/cpp/src/TensorflowOperators/CudaRenderer/CudaRenderer.cpp:25-26).

Shape: the icosphere subdivision-5 character (10,242 vertices / 20,480
triangles) skinned per vertex by dual quaternions of a 24-joint tree, 2
frames x 8 cameras whose sizes cover {512x512, 768x1024, 1024x1024,
1536x1024} twice (fx = fy = 600 min(W, H) / 512), vertex-colour raster with
the masked L1, projection, mesh boundary and silhouette DT loss, adjoints to
the joint angles and the vertex colours, parity-mode renderer adjoint.

Per camera, on the chain's own upstream buffers: face buffer bit-exact
outside quantised-depth ties, boundary flags and silhouette outputs
bit-identical; summed over cameras: losses, vertex-position, vertex-colour
and joint-angle gradients within 1e-5 norm-wise.  Also: the CUDA-graph
replay of the mixed-size step equals its eager run.
"""
import os

import numpy as np
import pytest
import torch

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.chain import DeformRenderChain, character
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
B = 2
SIZES = list(S.MIXED_SIZES) * 2
WS, HS = [w for w, _ in SIZES], [h for _, h in SIZES]
C = len(SIZES)
TOL = 1e-5


def nrel(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


@pytest.fixture(scope="module")
def run():
    sc = S.chain_scene(5, 200, 24, B, C, WS, HS, seed=11)
    ch = DeformRenderChain(sc, DEV, B, C, WS, HS, gradient_parity=True, deformation="dq")
    ch.step()
    torch.cuda.synchronize()
    return sc, ch


def cam_slices():
    off = 0
    for c in range(C):
        n = WS[c] * HS[c]
        yield c, off, n
        off += n


@pytest.mark.skipif(not (O.ref_available() and os.path.exists(O.REF_MB_LIB)),
                    reason="reference kernels (oracle/_ref) not built")
def test_c3_each_camera_matches_reference_kernels_at_its_size(run):
    sc, ch = run
    o, i = ch.buf, ch.inp
    # vertex DQ skinning: the reference kernel fed the device kinematics' dual quaternions
    skin = O.RefSkin(character(sc))
    v, n, _, _ = skin.dq_forward(o["dq"], o["weights"])
    assert nrel(o["v"], v) < 1e-6 and nrel(o["n"], n) < 1e-6
    ties = ch.rend.forward(o["v"], i["colors"], i["texture"], i["sh"], i["extr"], i["intr"], diagnostics=True)[6]
    # the fused L1's gradient image: normalised by the nonzero differences of the whole call
    diff = 255.0 * o["render"] - 255.0 * i["target"]
    diff = diff * (o["face"] >= 0).unsqueeze(-1)
    cnt = int(torch.count_nonzero(diff))
    gimg = 255.0 * torch.sign(diff) / cnt
    l1 = float(diff.double().abs().sum() / cnt)
    s = O.RefSilhouette()
    gv = torch.zeros_like(o["gv"], dtype=torch.float64)
    gcol = torch.zeros_like(gv)
    sil0 = sil1 = 0.0
    for c, off, npx in cam_slices():
        W, H = WS[c], HS[c]
        ex, it = i["extr"][:, 12 * c:12 * c + 12].contiguous(), i["intr"][:, 9 * c:9 * c + 9].contiguous()
        sh = i["sh"][:, c:c + 1].contiguous()
        sl = lambda t, k=(): t[:, off:off + npx].reshape((B, 1, H, W) + k).contiguous()  # noqa: E731
        r = O.RefRenderer(sc["faces"], sc["texcoords"], ch.N, 1, W, H, "vertexColor", "shadeless", "none", 2, 2)
        fw = r.forward(B, o["v"], i["colors"], i["texture"], sh, ex, it, depth=False)
        face = sl(o["face"])
        mism = face != fw["face"]
        assert int((fw["face"] >= 0).sum()) > 1000, c
        assert not bool((mism & (sl(ties) < 2)).any()), (c, int((mism & (sl(ties) < 2)).sum()))
        # the adjoint on the chain's own forward buffers
        vn = o["vnormal"][:, c:c + 1].contiguous()
        bw = r.backward(B, sl(gimg, (3,)), o["v"], i["colors"], i["texture"], sh, sl(i["target"], (3,)), vn,
                        sl(o["bary"], (2,)), face, ex, it)
        gv += bw["vertex_pos_grad"].double()
        gcol += bw["vertex_color_grad"].double()
        # projection, boundary and silhouette at this camera's size
        p2d = s.project(o["v"], None, ex, it, 1)
        n2d = s.project(o["v"], o["n"], ex, it, 0)
        assert torch.equal(p2d, o["p2d"][:, c:c + 1]) and torch.equal(n2d, o["n2d"][:, c:c + 1]), c
        isb = O.ref_mesh_boundary(sc["faces"], o["v"], ex, it, W, H)
        assert torch.equal(isb, o["isb"][:, c:c + 1]), c
        assert int(isb.sum()) > 0, c
        # the reference op reads the distance image as [B, C, U, V] with rows of U = W values
        dt = i["dt"][:, off:off + npx].reshape(B, 1, W, H).contiguous()
        crops = i["crops"][:, c:c + 1].contiguous()
        res, res1, dtg, cid = s.forward(p2d, n2d, isb, dt, crops)
        assert torch.equal(res, o["res"][:, c:c + 1]), c
        assert torch.equal(res1, sl(o["res1"], (2,))), c
        assert torch.equal(dtg, o["dtg"][:, c:c + 1]), c
        assert torch.equal(cid, sl(o["cid"])), c
        gp = s.backward(2 * ch.w_sil * res, 2 * ch.w_sil1 * res1, dtg, cid, crops)
        gv += s.project_grad(gp, o["v"], ex, it, 1).double()
        sil0 += float((res.double() ** 2).sum())
        sil1 += float((res1.double() ** 2).sum())
    loss = torch.tensor([l1, ch.w_sil * sil0, ch.w_sil1 * sil1], dtype=torch.float64)
    assert nrel(ch.loss, loss) < TOL, (ch.loss, loss)
    assert nrel(o["gcol"], gcol) < TOL
    assert nrel(o["gv"], gv) < TOL
    # joint angles: the reference DQ adjoint on the summed vertex gradient
    gd, _ = skin.dq_backward(gv.float().contiguous(), o["v"], o["gjp"], o["gja"], o["dq"], o["weights"],
                             sc["skin_weights"])
    assert nrel(o["gdofs"], gd) < TOL, nrel(o["gdofs"], gd)


def test_c3_graph_replay_matches_eager(run):
    sc, ch = run
    eager = {k: ch.buf[k].clone() for k in ("face", "render", "isb", "res1", "cid", "gdofs", "gcol", "gv")}
    loss = ch.loss.clone()
    g = ch.capture_step()
    for k in eager:
        ch.buf[k].zero_()
    g.replay()
    torch.cuda.synchronize()
    for k in ("face", "render", "isb", "res1", "cid"):
        assert torch.equal(ch.buf[k], eager[k]), k
    for k in ("gdofs", "gcol", "gv"):  # float atomics: equal up to summation order
        assert nrel(ch.buf[k], eager[k]) < 1e-5, k
    assert nrel(ch.loss, loss) < 1e-6
    assert float(ch.buf["gdofs"].abs().sum()) > 0
