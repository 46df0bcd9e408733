"""ARAP regulariser host side: the synthetic node graph and the FP64
oracle's adjoint against finite differences (no GPU)."""
import numpy as np

from deepcharacters_b200 import synthetic as S
from oracle import arap_oracle as AO


def _scene(seed=3):
    sc = S.eg_scene(1, 20, batch=2, seed=seed, n_markers=0)
    ng = S.node_graph(sc["verts"], sc["graph"], 3, np.random.default_rng(seed))
    return sc, ng


def test_node_graph_is_symmetric_sorted_and_weighted():
    sc, ng = _scene()
    M = sc["graph"].n_nodes
    lists = [list(ng.n2n_indices[o:o + n]) for o, n in zip(ng.n2n_offsets, ng.n2n_sizes)]
    for j, L in enumerate(lists):
        assert L == sorted(L) and j not in L and len(set(L)) == len(L)
        for k in L:
            assert j in lists[k]
    assert ng.max_connections == max(len(L) for L in lists) and len(lists) == M
    # rigidity = mean segmentation weight over each node's vertex connections
    seg = np.random.default_rng(1).uniform(1.0, 40.0, sc["verts"].shape[0]).astype(np.float32)
    g = sc["graph"]
    for refinement in (False, True):
        r = S.node_graph(sc["verts"], g, 3, np.random.default_rng(0), refinement, seg).rigidity
        v = np.repeat(np.arange(sc["verts"].shape[0]), g.v2n_sizes)
        w = seg[v].astype(np.float64)
        if refinement:
            w = np.where(w < 20.0, w / 10.0, w)
        want = np.bincount(g.v2n_indices, w, M) / np.bincount(g.v2n_indices, minlength=M)
        assert np.allclose(r, want, rtol=1e-5)


def test_oracle_adjoint_matches_finite_differences():
    """For a symmetric graph the reference's adjoint is the exact gradient of
    sum(c * nodes_arap_loss)."""
    sc, ng = _scene(5)
    args = (sc["verts"], sc["graph"].node_vertex, ng.n2n_offsets, ng.n2n_sizes, ng.n2n_indices)
    rng = np.random.default_rng(2)
    T = rng.normal(0, 5.0, sc["dT"].shape)
    A = rng.normal(0, 0.3, sc["dA"].shape)
    loss, _, _ = AO.arap_forward(*args, ng.rigidity, ng.max_connections, T, A)
    c = rng.normal(size=loss.shape)
    gT, gA = AO.arap_backward(*args, ng.max_connections, c, A)

    def f(T, A):
        return float((AO.arap_forward(*args, ng.rigidity, ng.max_connections, T, A)[0] * c).sum())
    for X, G, h in ((T, gT, 1e-3), (A, gA, 1e-6)):
        for idx in [(0, 1, 0), (1, 7, 2), (0, 19, 1)]:
            Xp, Xm = X.copy(), X.copy()
            Xp[idx] += h
            Xm[idx] -= h
            fd = (f(Xp, A) - f(Xm, A)) / (2 * h) if X is T else (f(T, Xp) - f(T, Xm)) / (2 * h)
            assert abs(fd - G[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, G[idx])
