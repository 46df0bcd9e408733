"""The deform-and-render chain at the benchmark's per-frame shape, checked
against the reference kernels and the FP64 oracle.

Shape: icosphere subdivision 6 (40,962 vertices / 81,920 triangles, radius
1000 mm, 10 mm jitter), a 1000-node embedded graph (K = 4), a 24-joint tree
with 3 revolute dofs per joint, one frame seen by 4 cameras at 1024 x 1024 on
a 3 m ring (fx = fy = 1200), vertex-colour raster with the masked L1 image
loss, projection + mesh boundary + silhouette DT loss, and the adjoints to
node rotations / translations, vertex colours and joint angles -- the chain
``bench.py`` times, with its default tiling (8-px tiles, 256-entry bins).

Two comparisons:
* parity mode (the reference's barycentric-Jacobian formula) against the
  same composition of the reference kernels (oracle/chain_ref.py): face
  buffer bit-exact outside quantised-depth ties, losses and gradients within
  1e-5 norm-wise;
* both adjoint modes (the parity mode and the closed form) against the FP64
  oracle on the same forward buffers, on all pixels and on the
  well-conditioned ones, and the joint-angle gradient (no reference
  counterpart) against FP64 central differences.

With HC_PARITY_RECORD=<file> set, the measured errors are written there as
JSON (the benchmark line quotes the committed record).
"""
import json
import os

import numpy as np
import pytest
import torch

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.chain import DeformRenderChain, character, eg_data
from deepcharacters_b200.renderer import renderer_backward
from oracle import oracle as O
from oracle import skinning_oracle as K

from _conditioning import well_conditioned_mask

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
B, C, RES, FX = 1, 4, 1024, 1200.0
TOL = 1e-5


def nrel(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


def record(section, values):
    path = os.environ.get("HC_PARITY_RECORD")
    print(section, json.dumps(values))
    if not path:
        return
    rec = {}
    if os.path.exists(path):
        with open(path) as fh:
            rec = json.load(fh)
    rec[section] = values
    with open(path, "w") as fh:
        json.dump(rec, fh, indent=1, sort_keys=True)


@pytest.fixture(scope="module")
def scene():
    return S.chain_scene(6, 1000, 24, B, C, RES, RES, seed=2, fx=FX)


@pytest.mark.skipif(not (O.ref_available() and os.path.exists(O.REF_MB_LIB)),
                    reason="reference kernels (oracle/_ref) not built")
def test_c2_parity_mode_matches_reference_kernels(scene):
    from oracle.chain_ref import RefChain
    ours = DeformRenderChain(scene, DEV, B, C, RES, RES, gradient_parity=True, joint_gradients=True)
    ours.step()
    torch.cuda.synchronize()
    o = ours.buf
    ref = RefChain(scene, DEV, B, C, RES, RES)
    r0 = ref.step()  # host node skinning, the reference's CPU op
    e = {"node_translation": nrel(o["sT"], r0["sT"])}
    d = (o["sA"] - r0["sA"]).double()
    e["node_rotation_max_abs"] = float(torch.atan2(torch.sin(d), torch.cos(d)).abs().max())
    r1 = ref.step(sT=o["sT"], sA=o["sA"])  # EG on identical node transforms
    e["eg_vertices"] = nrel(o["v"], r1["v"])
    e["eg_normals"] = nrel(o["n"], r1["n"])
    raster = dict(bary=o["bary"], face=o["face"], render=o["render"], vnormal=o["vnormal"])
    r = ref.step(sT=o["sT"], sA=o["sA"], verts=o["v"], normals=o["n"], raster=raster)
    torch.cuda.synchronize()
    covered = r["face"] >= 0
    ties = ours.rend.forward(o["v"], ours.inp["colors"], ours.inp["texture"], ours.inp["sh"], ours.inp["extr"],
                             ours.inp["intr"], diagnostics=True)[6]
    mism = o["face"] != r["face"]
    e["covered_pixels"] = int(covered.sum())
    e["tie_pixels"] = int((ties >= 2).sum())
    e["face_mismatch_outside_ties"] = int((mism & (ties < 2)).sum())
    e["face_mismatch_at_ties"] = int((mism & (ties >= 2)).sum())
    e["boundary_flags_equal"] = bool(torch.equal(o["isb"], r["isb"]))
    for k in ("loss", "gcol", "gv_sil", "gv", "gT", "gA"):
        e[k] = nrel(ours.loss if k == "loss" else o[k], r[k])
    record("parity_mode_vs_reference_kernels", e)
    assert e["covered_pixels"] > 100000
    assert e["face_mismatch_outside_ties"] == 0
    assert e["boundary_flags_equal"] and int(r["isb"].sum()) > 0
    assert e["node_translation"] < 1e-5 and e["node_rotation_max_abs"] < 1e-4
    assert e["eg_vertices"] < 1e-6 and e["eg_normals"] < 1e-6
    for k in ("loss", "gcol", "gv_sil", "gv", "gT", "gA"):
        assert e[k] < TOL, (k, e[k])


def test_c2_adjoints_against_fp64(scene):
    """Both adjoint modes against the FP64 oracle, silhouette weights 0 so
    that the vertex gradient is the raster adjoint alone: the oracle's raster
    adjoint of the same L1 image gradient on the same forward buffers (all
    pixels, and the well-conditioned ones), then the EG adjoint (full skinned
    gradients) of the FP64 vertex gradient, and the node-skinning adjoint
    against central differences.  The closed form must meet 1e-5 on the
    well-conditioned pixels (or stay within the FP32 floor of the reference
    formula); the parity mode's numbers are that floor and are recorded."""
    sc = scene
    rec = {}
    o64s = {}
    d = eg_data(sc)
    for mode in ("exact", "parity"):
        ours = DeformRenderChain(sc, DEV, B, C, RES, RES, w_sil=0.0, w_sil1=0.0, gradient_parity=mode == "parity",
                                 joint_gradients=True)
        ours.step()
        torch.cuda.synchronize()
        o = {k: (v.cpu().numpy() if v is not None else None) for k, v in ours.buf.items()}
        face, bary, render = o["face"], o["bary"], o["render"]
        diff = np.float32(255.0) * render - np.float32(255.0) * sc["target"].astype(np.float32)
        diff = diff * (face >= 0)[..., None]
        cnt = int(np.count_nonzero(diff))
        gimg = (np.sign(diff) * (np.float32(255.0) / np.float32(cnt))).astype(np.float32)
        l1 = float(np.abs(diff.astype(np.float64)).sum() / cnt)
        if not o64s:  # the forward does not depend on the adjoint mode: one FP64 reference
            mask = well_conditioned_mask(o["v"], sc["faces"], sc["texcoords"], sc["texture"].shape[1], sc["extr"],
                                         sc["intr"], face, bary, "vertexColor")
            rec["well_conditioned_fraction"] = float(mask[face >= 0].mean())
            for name, g in (("all_pixels", gimg), ("well_conditioned_pixels", gimg * mask[..., None])):
                args = (sc["faces"], sc["texcoords"], B, C, RES, RES, "vertexColor", "shadeless", g, o["v"],
                        sc["colors"], sc["texture"], sc["sh"], sc["target"], o["vnormal"], bary, face, sc["extr"],
                        sc["intr"])
                o64s[name] = (g, O.render_backward(*args, ifs=2, tfs=2, precision="f64"),
                              O.render_backward(*args, ifs=2, tfs=2, precision="f32"))
            base = (face.copy(), render.copy())
        assert np.array_equal(face, base[0]) and np.array_equal(render, base[1])
        e = {"l1_loss": abs(float(ours.loss[0]) - l1) / l1}
        for name, (g, o64, o32) in o64s.items():
            if name == "all_pixels":
                gv, gcol = o["gv"], o["gcol"]
            else:  # the same adjoint on the masked image gradient
                gpos_t, gcol_t, _, _ = renderer_backward(
                    ours.rend, torch.from_numpy(g).to(DEV), ours.buf["v"], ours.inp["colors"], ours.inp["texture"],
                    ours.inp["sh"], ours.inp["target"], ours.buf["vnormal"], ours.buf["bary"], ours.buf["face"],
                    ours.inp["extr"], ours.inp["intr"])
                gv, gcol = gpos_t.cpu().numpy(), gcol_t.cpu().numpy()
            r = {"vertex_positions": nrel(gv, o64["vertex_pos_grad"]),
                 "vertex_colours": nrel(gcol, o64["vertex_color_grad"]),
                 "reference_formula_fp32_positions": nrel(o32["vertex_pos_grad"], o64["vertex_pos_grad"])}
            if name == "all_pixels":
                eb = O.eg_backward(d, o64["vertex_pos_grad"], np.zeros((B, len(sc["markers"]), 3), np.float32),
                                   sc["dT"], sc["dA"], o["sA"], sc["disp"], full=True, precision="f64")
                r.update(node_translations=nrel(o["gT"], eb["t"]), node_rotations=nrel(o["gA"], eb["r"]),
                         skinned_translations=nrel(o["gsT"], eb["st"]), skinned_rotations=nrel(o["gsA"], eb["sr"]))
            e[name] = r
        rec[mode] = e
        if mode == "exact":
            # joint angles: the node-skinning adjoint of our (gsT, gsA) against
            # FP64 central differences of the node-skinning restatement
            ch = character(sc)
            dofs = sc["dofs"].astype(np.float64)
            nodes = sc["graph"].node_vertex
            gsT, gsA = o["gsT"].astype(np.float64), o["gsA"].astype(np.float64)

            def loss(dd):
                t, a, _ = K.pose2eg(ch, dd, nodes, sc["skin_weights"])
                return (gsT * t).sum(axis=(1, 2)) + (gsA * a).sum(axis=(1, 2))

            h = 1e-6
            fd = np.zeros_like(dofs)
            for k in range(dofs.shape[1]):
                p, m = dofs.copy(), dofs.copy()
                p[:, k] += h
                m[:, k] -= h
                fd[:, k] = (loss(p) - loss(m)) / (2 * h)
            rec["joint_angles_vs_fp64_central_differences"] = nrel(o["gdofs"], fd)
        del ours
    record("adjoints_vs_fp64", rec)
    for mode in ("exact", "parity"):
        assert rec[mode]["l1_loss"] < 1e-5
        assert rec[mode]["all_pixels"]["vertex_colours"] < TOL
    w = rec["exact"]["well_conditioned_pixels"]
    assert w["vertex_positions"] < max(TOL, 1.25 * w["reference_formula_fp32_positions"]), w
    assert w["vertex_colours"] < TOL, w
    a = rec["exact"]["all_pixels"]
    assert a["node_translations"] < 1e-3 and a["node_rotations"] < 1e-3, a
    assert rec["joint_angles_vs_fp64_central_differences"] < 1e-4
