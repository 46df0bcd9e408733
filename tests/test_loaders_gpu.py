"""Device ops built from loaded character and graph files.

The files are written in the reference's formats by ``test_loaders_cpu``;
skinning (with non-unit joint scales), the embedded graph and the ARAP
regulariser then run on the GPU from the loaded arrays and are compared with
the FP64 oracle and the reference kernels."""
import numpy as np
import pytest
import torch

from deepcharacters_b200 import loaders as L
from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.arap import ArapEngine
from deepcharacters_b200.embedded_graph import EmbeddedGraphEngine, EmbeddedGraphGpu
from deepcharacters_b200.skinning import SkinningEngine
from oracle import oracle as O
from oracle import skinning_oracle as K
from test_loaders_cpu import write_character

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference kernels (oracle/_ref) not built")


def tmp_graph(cf):
    import os
    return os.path.join(os.path.dirname(cf.path), "graph.obj")


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(DEV)


def nrel(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


@pytest.fixture(scope="module")
def loaded(tmp_path_factory):
    d = tmp_path_factory.mktemp("character")
    sc = S.skinning_scene(3, 12, batch=2, seed=29)
    J = sc["skeleton"].n_joints
    scales = (1.0 + 0.02 * np.arange(J)).astype(np.float32)
    gv, gf = S.icosphere(1)
    seg = np.random.default_rng(3).choice([0, 9, 14], size=sc["verts"].shape[0])
    path = write_character(str(d), sc, scales=scales, segmentation=seg, graph=((gv * 980.0).astype(np.float32), gf),
                           markers=[("j00_z", (0.0, 10.0, 0.0)), ("j05_z", (3.0, 0.0, -4.0))])
    cf = L.load_character(path)
    return sc, cf, L.load_graph(cf, str(d / "graph.obj"))


def test_dq_skinning_of_a_loaded_scaled_character(loaded):
    sc, cf, _ = loaded
    ch = cf.character()
    assert not np.all(ch.joint_scale == 1.0)
    eng = SkinningEngine(ch)
    w = np.tile(cf.skin_weight[None], (2, 1, 1))
    v, n, gp, ga, dq, _ = eng.dq_forward(_t(sc["dofs"]), _t(w))
    _, _, gpos, gaxis = K.fk(ch, sc["dofs"])
    assert nrel(gp, gpos) < 1e-5 and nrel(ga, gaxis) < 1e-5
    dq_o = K.dual_quaternions(ch, sc["dofs"])
    # translation parts reach ~150 mm here: FP32 relative, not absolute, error
    assert nrel(dq[..., :4], dq_o[..., :4]) < 1e-6 and nrel(dq, dq_o) < 1e-6
    vo, no = K.dq_skin(ch, dq_o, w)
    assert nrel(v, vo) < 1e-5 and nrel(n, no) < 1e-5
    # at the bind pose the skinned mesh is the base mesh scaled about each joint:
    # with unit scales it is the base mesh itself
    ch1 = cf.character()
    ch1.joint_scale = np.ones_like(ch1.joint_scale)
    ch1.skin_scale = np.ones_like(ch1.skin_scale)
    v0 = SkinningEngine(ch1).dq_forward(_t(np.zeros((1, ch.n_dofs))), _t(w[:1]))[0]
    assert nrel(v0, ch1.base_vertices[None]) < 1e-6


@needs_ref
def test_embedded_graph_from_loaded_files_matches_reference_kernels(loaded):
    sc, cf, g = loaded
    d = g.eg
    M = d.node_vertex.shape[0]
    rng = np.random.default_rng(7)
    ins = [_t(rng.normal(0, s, (2, M, 3))) for s in (5.0, 0.05, 5.0, 0.1)]
    ins.append(_t(rng.normal(0, 1.0, (2, d.base_vertices.shape[0], 3))))
    ours = EmbeddedGraphEngine(d).forward(*ins)
    op = EmbeddedGraphGpu(cf.path, str(tmp_graph(cf)), 2, *ins).getNode()
    for a, b in zip(op, ours):
        assert torch.equal(a, b)
    ref = O.RefEG(d, DEV).forward(*ins)
    torch.cuda.synchronize()
    assert nrel(ours[0], ref["vertices"]) < 1e-7
    assert nrel(ours[1], ref["normals"]) < 1e-6
    assert nrel(ours[3], ref["graph"]) < 1e-7
    assert ours[2].shape[1] == 2


@needs_ref
def test_arap_from_loaded_graph_matches_reference_kernels(loaded):
    _, cf, g = loaded
    args = (g.eg.base_vertices, g.eg.node_vertex, g.n2n_offsets, g.n2n_sizes, g.n2n_indices, g.rigidity,
            g.max_connections)
    rng = np.random.default_rng(9)
    M = g.eg.node_vertex.shape[0]
    T, A = _t(rng.normal(0, 8.0, (2, M, 3))), _t(rng.normal(0, 0.4, (2, M, 3)))
    ours = ArapEngine.from_graph_file(g).forward(T, A)
    theirs = O.RefArap(*args, DEV).forward(T, A)
    torch.cuda.synchronize()
    for a, b in zip(ours, theirs):
        assert torch.equal(a, b)
