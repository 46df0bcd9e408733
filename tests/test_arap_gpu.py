"""ARAP regulariser on the GPU against the reference kernels (oracle/_ref)
and the FP64 oracle."""
import numpy as np
import pytest
import torch

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.arap import ArapEngine, embedded_graph_arap
from oracle import arap_oracle as AO
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference kernels (oracle/_ref) not built")


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV, torch.float32)


def nrel(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


@pytest.fixture(scope="module")
def scene():
    sc = S.eg_scene(3, 300, batch=3, seed=41, n_markers=0)
    ng = S.node_graph(sc["verts"], sc["graph"], 6, np.random.default_rng(42))
    rng = np.random.default_rng(43)
    T = rng.normal(0, 8.0, sc["dT"].shape).astype(np.float32)
    A = rng.normal(0, 0.4, sc["dA"].shape).astype(np.float32)
    return sc, ng, T, A


def _graph(sc, ng):
    return (sc["verts"], sc["graph"].node_vertex, ng.n2n_offsets, ng.n2n_sizes, ng.n2n_indices, ng.rigidity,
            ng.max_connections)


@needs_ref
def test_arap_matches_reference_kernels(scene):
    sc, ng, T, A = scene
    g = _graph(sc, ng)
    eng = ArapEngine(*g)
    ref = O.RefArap(*g, DEV)
    ours = eng.forward(_t(T), _t(A))
    theirs = ref.forward(_t(T), _t(A))
    torch.cuda.synchronize()
    for a, b, name in zip(ours, theirs, ("loss", "weights", "rotation")):
        assert torch.equal(a, b), (name, nrel(a, b))
    G = torch.randn(ours[0].shape, device=DEV, generator=torch.Generator(DEV).manual_seed(1))
    for a, b in zip(eng.backward(G, ours[2]), ref.backward(G, theirs[2])):
        assert nrel(a, b) < 1e-6


@needs_ref
def test_arap_asymmetric_graph_matches_reference_kernels(scene):
    """One-way and repeated neighbours: the translation adjoint takes the
    neighbour's last slot that names the node, or none."""
    sc, ng, T, A = scene
    lists = [list(ng.n2n_indices[o:o + n]) for o, n in zip(ng.n2n_offsets, ng.n2n_sizes)]
    lists[0] = lists[0][:-1]            # 0 drops its last neighbour, which still lists 0
    lists[5] = lists[5] + [lists[5][0]]  # a repeated neighbour
    lists[9] = []                        # a node without neighbours
    sizes = np.array([len(x) for x in lists], np.int32)
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int32)
    idx = np.array([q for x in lists for q in x], np.int32)
    g = (sc["verts"], sc["graph"].node_vertex, offs, sizes, idx, ng.rigidity, int(sizes.max()))
    eng, ref = ArapEngine(*g), O.RefArap(*g, DEV)
    ours, theirs = eng.forward(_t(T), _t(A)), ref.forward(_t(T), _t(A))
    assert all(torch.equal(a, b) for a, b in zip(ours, theirs))
    G = torch.randn(ours[0].shape, device=DEV, generator=torch.Generator(DEV).manual_seed(2))
    for a, b in zip(eng.backward(G, ours[2]), ref.backward(G, theirs[2])):
        assert nrel(a, b) < 1e-6


def test_arap_matches_fp64_oracle_and_autograd(scene):
    sc, ng, T, A = scene
    g = _graph(sc, ng)
    eng = ArapEngine(*g)
    Tt, At = _t(T).requires_grad_(True), _t(A).requires_grad_(True)
    loss, w, rot = embedded_graph_arap(eng, Tt, At)
    ol, ow, _ = AO.arap_forward(*g[:6], g[6], T, A)
    assert nrel(loss.detach(), ol) < 1e-6 and nrel(w, ow) < 1e-7
    c = torch.randn(loss.shape, device=DEV, generator=torch.Generator(DEV).manual_seed(3))
    (loss * c).sum().backward()
    oT, oA = AO.arap_backward(*g[:5], g[6], c.cpu().numpy(), A)
    assert nrel(Tt.grad, oT) < 1e-6
    assert nrel(At.grad, oA) < 1e-5
