"""Generate the golden vectors of this directory from the reference's own
kernels (oracle/_ref, compiled from the reference tree; needs a GPU).

    python tests/golden/make_golden.py [out_dir]

Each fixture is a small seeded case (inputs and the reference kernels'
outputs) saved as .npz.  tests/test_golden_cpu.py checks the CPU oracle
against them without a GPU, which pins the oracle to the reference.
"""
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from deepcharacters_b200 import synthetic as S  # noqa: E402
from deepcharacters_b200.embedded_graph import EGData  # noqa: E402
from deepcharacters_b200.skinning import Character  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle import silhouette_oracle as SO  # noqa: E402
from oracle import skinning_oracle as K  # noqa: E402

DEV = "cuda:0"


def t(a, dt=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV, dt)


def n(x):
    return x.detach().cpu().numpy()


def render(out):
    sc = S.render_scene(2, batch=1, views=2, width=64, height=48, seed=3, texture_size=16)
    keep = {k: sc[k] for k in ("faces", "texcoords", "verts", "colors", "texture", "sh", "extr", "intr", "target")}
    g = np.random.default_rng(5).normal(size=(1, 2, 48, 64, 3)).astype(np.float32)
    for albedo, shading in (("vertexColor", "shaded"), ("textured", "shadeless")):
        ref = O.RefRenderer(sc["faces"], sc["texcoords"], sc["N"], 2, 64, 48, albedo, shading)
        fw = ref.forward(1, t(sc["verts"]), t(sc["colors"]), t(sc["texture"]), t(sc["sh"]), t(sc["extr"]),
                         t(sc["intr"]))
        bw = ref.backward(1, t(g), t(sc["verts"]), t(sc["colors"]), t(sc["texture"]), t(sc["sh"]), t(sc["target"]),
                          fw["vnormal"], fw["bary"], fw["face"], t(sc["extr"]), t(sc["intr"]))
        np.savez_compressed(os.path.join(out, f"render_{albedo}_{shading}.npz"), render_grad=g, **keep,
                            **{f"out_{k}": n(v) for k, v in fw.items() if v is not None},
                            **{f"grad_{k}": n(v) for k, v in bw.items()})


def eg(out):
    sc = S.eg_scene(2, 30, batch=1, seed=7, n_markers=4)
    d = EGData.from_synthetic(sc["verts"], sc["faces"], sc["graph"], sc["markers"], sc["marker_node"])
    ins = [t(sc[k]) for k in ("dT", "dA", "sT", "sA", "disp")]
    ref = O.RefEG(d, DEV)
    fw = ref.forward(*ins)
    rng = np.random.default_rng(8)
    gv = rng.normal(size=(1, d.base_vertices.shape[0], 3)).astype(np.float32)
    gm = rng.normal(size=(1, 4, 3)).astype(np.float32)
    bw = ref.backward(t(gv), t(gm), ins[1], ins[3])
    g = sc["graph"]
    np.savez_compressed(os.path.join(out, "eg.npz"), base=d.base_vertices, faces=d.faces, markers=sc["markers"],
                        marker_node=sc["marker_node"], node_vertex=g.node_vertex, v2n_offsets=g.v2n_offsets,
                        v2n_sizes=g.v2n_sizes, v2n_indices=g.v2n_indices, v2n_weights=g.v2n_weights,
                        n2v_offsets=g.n2v_offsets, n2v_sizes=g.n2v_sizes, n2v_indices=g.n2v_indices,
                        n2v_weights=g.n2v_weights, dT=sc["dT"], dA=sc["dA"], sT=sc["sT"], sA=sc["sA"], disp=sc["disp"],
                        gv=gv, gm=gm, **{f"out_{k}": n(v) for k, v in fw.items()},
                        **{f"grad_{k}": n(v) for k, v in bw.items()})


def skin(out):
    sc = S.skinning_scene(2, 4, batch=1, seed=9)
    ch = Character.from_synthetic(sc["skeleton"], sc["verts"], sc["faces"], sc["skin_index"])
    dq = K.dual_quaternions(ch, sc["dofs"]).astype(np.float32)
    _, _, gpos, gaxis = K.fk(ch, sc["dofs"])
    ref = O.RefSkin(ch)
    w = t(sc["weights"])
    rv, rn, rdq, rw = ref.dq_forward(t(dq), w)
    g = np.random.default_rng(10).normal(size=(1, ch.base_vertices.shape[0], 3)).astype(np.float32)
    rgd, rgw = ref.dq_backward(t(g), rv, t(gpos.astype(np.float32)), t(gaxis.astype(np.float32)), t(dq), w,
                               sc["weights"][0])
    sk = sc["skeleton"]
    np.savez_compressed(os.path.join(out, "dq_skinning.npz"), verts=sc["verts"], faces=sc["faces"],
                        skin_index=sc["skin_index"], weights=sc["weights"], dofs=sc["dofs"], dq=dq,
                        gpos=gpos.astype(np.float32), gaxis=gaxis.astype(np.float32), grad=g,
                        parent=sk.parent, offset=sk.offset, axis=sk.axis, dof_joint=sk.dof_joint,
                        dof_weight=sk.dof_weight, skin_joint=sk.skin_joint,
                        out_vertices=n(rv), out_normals=n(rn), grad_dofs=n(rgd), grad_weights=n(rgw))


def silhouette(out):
    sc = S.render_scene(2, batch=1, views=2, width=64, height=64, seed=13)
    v = sc["verts"].astype(np.float64)
    normals = (v / np.linalg.norm(v, axis=2, keepdims=True)).astype(np.float32)
    rs = O.RefSilhouette()
    p2d = rs.project(t(sc["verts"]), None, t(sc["extr"]), t(sc["intr"]), 1)
    n2d = rs.project(t(sc["verts"]), t(normals), t(sc["extr"]), t(sc["intr"]), 0)
    isb = O.ref_mesh_boundary(sc["faces"], t(sc["verts"]), t(sc["extr"]), t(sc["intr"]), 64, 64)
    dt = S.silhouette_masks(1, 2, 64, 64, seed=14, scale=64 / 512)
    crops = S.identity_crops(1, 2, 64, 64)
    res, res1, dtg, cid = rs.forward(p2d, n2d, isb, t(dt, torch.uint8), t(crops))
    rng = np.random.default_rng(15)
    g = rng.normal(size=n(res).shape).astype(np.float32)
    g1 = rng.normal(size=n(res1).shape).astype(np.float32)
    gp = rs.backward(t(g), t(g1), dtg, cid, t(crops))
    np.savez_compressed(os.path.join(out, "silhouette.npz"), verts=sc["verts"], normals=normals, faces=sc["faces"],
                        extr=sc["extr"], intr=sc["intr"], dt=dt, crops=crops, g=g, g1=g1, out_p2d=n(p2d),
                        out_n2d=n(n2d), out_isb=n(isb), out_res=n(res), out_res1=n(res1), out_dtg=n(dtg),
                        out_cid=n(cid), grad_points=n(gp))


def uv(out):
    sc = S.render_scene(2, batch=1, views=1, width=32, height=32, seed=17, texture_size=32)
    res = {}
    for mode in ("normal", "position", "face"):
        o = O.RefUV(sc["faces"], sc["texcoords"], sc["N"], 1, 32, 32, mode).forward(
            1, t(sc["verts"]), t(sc["extr"]), t(sc["intr"]), 32, 32)
        res[f"out_{mode}"] = n(o["normal_map"])
        res["out_vnormal"] = n(o["vnormal"])
    np.savez_compressed(os.path.join(out, "uv_maps.npz"), faces=sc["faces"], texcoords=sc["texcoords"],
                        verts=sc["verts"], extr=sc["extr"], intr=sc["intr"], **res)


def arap(out):
    sc = S.eg_scene(2, 40, batch=2, seed=21, n_markers=0)
    ng = S.node_graph(sc["verts"], sc["graph"], 4, np.random.default_rng(22))
    ref = O.RefArap(sc["verts"], sc["graph"].node_vertex, ng.n2n_offsets, ng.n2n_sizes, ng.n2n_indices, ng.rigidity,
                    ng.max_connections, DEV)
    T = (sc["dT"] * 3.0).astype(np.float32)
    A = (sc["dA"] * 4.0).astype(np.float32)
    loss, w, rot = ref.forward(t(T), t(A))
    g = np.random.default_rng(23).normal(size=tuple(loss.shape)).astype(np.float32)
    gT, gA = ref.backward(t(g), rot)
    np.savez_compressed(os.path.join(out, "arap.npz"), base=sc["verts"], node_vertex=sc["graph"].node_vertex,
                        off=ng.n2n_offsets, size=ng.n2n_sizes, idx=ng.n2n_indices, rigid=ng.rigidity,
                        maxc=ng.max_connections, T=T, A=A, g=g, out_loss=n(loss), out_w=n(w), out_rot=n(rot),
                        grad_T=n(gT), grad_A=n(gA))


if __name__ == "__main__":
    out = sys.argv[1] if len(sys.argv) > 1 else HERE
    only = set(sys.argv[2:])  # optional: names of the fixtures to (re)make
    os.makedirs(out, exist_ok=True)
    for fn in (render, eg, skin, silhouette, uv, arap):
        if only and fn.__name__ not in only:
            continue
        fn(out)
        print("wrote", fn.__name__)
