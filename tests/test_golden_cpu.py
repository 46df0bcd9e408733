"""The CPU oracle against golden vectors produced by the reference's own
kernels (tests/golden/*.npz, written by tests/golden/make_golden.py on a GPU
from oracle/_ref).  Runs without a GPU: this pins the oracle's restatement
of the reference to the reference itself."""
import os

import numpy as np
import pytest

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.embedded_graph import EGData
from deepcharacters_b200.skinning import Character
from oracle import oracle as O
from oracle import silhouette_oracle as SO
from oracle import skinning_oracle as K

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not generated (python tests/golden/make_golden.py on a GPU)")
    return dict(np.load(p))


def nrel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("albedo,shading", [("vertexColor", "shaded"), ("textured", "shadeless")])
def test_render_oracle_matches_reference_golden(albedo, shading):
    g = load(f"render_{albedo}_{shading}.npz")
    fw = O.render_forward(g["faces"], g["texcoords"], 1, 2, 64, 48, albedo, shading, g["verts"], g["colors"],
                          g["texture"], g["sh"], g["extr"], g["intr"])
    robust = (fw["fragile"] == 0) & (fw["tie_count"] < 2)
    assert robust.mean() > 0.95 and (g["out_face"] >= 0).sum() > 500
    assert np.array_equal(fw["face"][robust], g["out_face"][robust])
    same = robust & (fw["face"] == g["out_face"]) & (g["out_face"] >= 0)
    assert np.abs(fw["render"][same] - g["out_render"][same]).max() < 1e-4
    assert np.abs(fw["bary"][same] - g["out_bary"][same]).max() < 1e-4
    assert nrel(fw["vnormal"], g["out_vnormal"]) < 1e-6
    # adjoint on the reference's own forward buffers, FP64 reference formulas
    bw = O.render_backward(g["faces"], g["texcoords"], 1, 2, 64, 48, albedo, shading, g["render_grad"], g["verts"],
                           g["colors"], g["texture"], g["sh"], g["target"], g["out_vnormal"], g["out_bary"],
                           g["out_face"], g["extr"], g["intr"])
    assert nrel(bw["vertex_pos_grad"], g["grad_vertex_pos_grad"]) < 2e-3
    if albedo == "vertexColor":
        assert nrel(bw["vertex_color_grad"], g["grad_vertex_color_grad"]) < 1e-5
        assert nrel(bw["sh_coeff_grad"], g["grad_sh_coeff_grad"]) < 1e-5
    else:
        assert nrel(bw["texture_grad"], g["grad_texture_grad"]) < 1e-5


def test_eg_oracle_matches_reference_golden():
    g = load("eg.npz")
    graph = S.EmbeddedGraph(g["node_vertex"], g["v2n_offsets"], g["v2n_sizes"], g["v2n_indices"], g["v2n_weights"],
                            g["n2v_offsets"], g["n2v_sizes"], g["n2v_indices"], g["n2v_weights"])
    d = EGData.from_synthetic(g["base"], g["faces"], graph, g["markers"], g["marker_node"])
    fw = O.eg_forward(d, g["dT"], g["dA"], g["sT"], g["sA"], g["disp"], precision="f64d")
    assert nrel(fw["vertices"], g["out_vertices"]) < 1e-6
    assert nrel(fw["normals"], g["out_normals"]) < 1e-5
    assert nrel(fw["markers"], g["out_markers"]) < 1e-6
    assert nrel(fw["graph"], g["out_graph"]) < 1e-6
    bw = O.eg_backward(d, g["gv"], g["gm"], g["dT"], g["dA"], g["sA"], g["disp"], full=False)
    assert nrel(bw["t"], g["grad_t"]) < 1e-5
    assert nrel(bw["r"], g["grad_r"]) < 1e-5
    assert nrel(bw["disp"], g["grad_disp"]) < 1e-5


def test_dq_skinning_oracle_matches_reference_golden():
    g = load("dq_skinning.npz")
    sk = S.Skeleton(g["parent"], g["offset"], g["axis"], g["dof_joint"], g["dof_weight"], g["skin_joint"])
    ch = Character.from_synthetic(sk, g["verts"], g["faces"], g["skin_index"])
    v, nrm = K.dq_skin(ch, g["dq"], g["weights"])
    assert nrel(v, g["out_vertices"]) < 1e-6
    assert nrel(nrm, g["out_normals"]) < 1e-5
    gd = K.dof_grad_reference(ch, g["out_vertices"], g["grad"], g["weights"], g["gpos"], g["gaxis"])
    assert nrel(gd, g["grad_dofs"]) < 1e-5


def test_silhouette_oracle_matches_reference_golden():
    g = load("silhouette.npz")
    p2d = SO.project(g["verts"], None, g["extr"], g["intr"], True)
    assert nrel(p2d, g["out_p2d"]) < 1e-6
    # the vector mode differences two projected points one unit apart
    # (CameraProjectionGPUOp.cu:44-84): at this image size that difference is
    # ~0.03 px, so the reference's FP32 result carries ~1e-3 relative error
    n2d = SO.project(g["verts"], g["normals"], g["extr"], g["intr"], False)
    assert nrel(n2d, g["out_n2d"]) < 5e-3
    isb = SO.mesh_boundary(g["faces"], g["out_p2d"], 64, 64)
    assert (isb != g["out_isb"]).mean() < 1e-2 and g["out_isb"].sum() > 0
    # data terms on the reference's own projection and boundary flags
    res, res1, dtg, cid = SO.silhouette_forward(g["out_p2d"], g["out_n2d"], g["out_isb"], g["dt"], g["crops"])
    assert np.array_equal(cid, g["out_cid"])
    assert nrel(res, g["out_res"]) < 1e-5 and nrel(res1, g["out_res1"]) < 1e-5 and nrel(dtg, g["out_dtg"]) < 1e-5
    gp = SO.silhouette_backward(g["g"], g["g1"], g["out_dtg"], g["out_cid"], g["crops"])
    assert nrel(gp, g["grad_points"]) < 1e-5


def test_uv_table_matches_reference_golden():
    g = load("uv_maps.npz")
    tab = O.texel_table(g["texcoords"], 32, 32)
    ref_face = g["out_face"][0, :, :, 0]
    assert (tab[..., 0] != ref_face).mean() < 0.02
    # position map from the table, where the face agrees
    v = g["verts"][0].astype(np.float64)
    f = np.asarray(g["faces"]).reshape(-1, 3)
    same = tab[..., 0] == ref_face
    idx = tab[..., 0].astype(int)
    pos = (v[f[idx, 0]] * tab[..., 1:2] + v[f[idx, 1]] * tab[..., 2:3] + v[f[idx, 2]] * tab[..., 3:4])
    assert np.abs(pos[same] - g["out_position"][0][same]).max() < 1e-2


def test_arap_oracle_matches_reference_golden():
    from oracle import arap_oracle as AO
    z = load("arap.npz")
    args = (z["base"], z["node_vertex"], z["off"], z["size"], z["idx"])
    loss, w, rot = AO.arap_forward(*args, z["rigid"], int(z["maxc"]), z["T"], z["A"])
    assert nrel(loss, z["out_loss"]) < 1e-6
    assert np.array_equal(w.astype(np.float32), z["out_w"])
    assert np.array_equal(rot.astype(np.float32), z["out_rot"])
    gT, gA = AO.arap_backward(*args, int(z["maxc"]), z["g"], z["A"])
    assert nrel(gT, z["grad_T"]) < 1e-6
    assert nrel(gA, z["grad_A"]) < 1e-5
