"""Embedded-graph CPU oracle: FP32 vs FP64 agreement and finite-difference
checks of the adjoint (the reference gradient and the full skinned mode)."""
import numpy as np
import pytest

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.embedded_graph import EGData
from oracle import oracle as O


@pytest.fixture(scope="module")
def scene():
    sc = S.eg_scene(2, 24, batch=2, seed=7, n_markers=3)
    d = EGData.from_synthetic(sc["verts"], sc["faces"], sc["graph"], sc["markers"], sc["marker_node"])
    return sc, d


def test_f32_matches_f64(scene):
    sc, d = scene
    a = O.eg_forward(d, sc["dT"], sc["dA"], sc["sT"], sc["sA"], sc["disp"], precision="f64")
    b = O.eg_forward(d, sc["dT"], sc["dA"], sc["sT"], sc["sA"], sc["disp"], precision="f32")
    for k in ("vertices", "normals", "markers", "graph"):
        np.testing.assert_allclose(b[k], a[k], rtol=1e-5, atol=1e-3)


def _loss(d, sc, gv, gm, **over):
    x = {k: sc[k].astype(np.float64) for k in ("dT", "dA", "sT", "sA", "disp")}
    x.update(over)
    o = O.eg_forward(d, *(x[k].astype(np.float32) for k in ("dT", "dA", "sT", "sA", "disp")), precision="f64d")
    return float((o["vertices"].astype(np.float64) * gv).sum() + (o["markers"].astype(np.float64) * gm).sum())


@pytest.mark.parametrize("name,key,h", [("delta translation", "dT", 1e-2), ("delta rotation", "dA", 1e-4),
                                        ("skinned translation", "sT", 1e-2), ("skinned rotation", "sA", 1e-4),
                                        ("displacement", "disp", 1e-2)])
def test_adjoint_matches_central_differences(scene, name, key, h):
    sc, d = scene
    rng = np.random.default_rng(1)
    gv = rng.normal(size=sc["disp"].shape)
    gm = rng.normal(size=(2, 3, 3))
    g = O.eg_backward(d, gv.astype(np.float32), gm.astype(np.float32), sc["dT"], sc["dA"], sc["sA"], sc["disp"],
                      full=True)
    ana = {"dT": g["t"], "dA": g["r"], "sT": g["st"], "sA": g["sr"], "disp": g["disp"]}[key]
    base = sc[key].astype(np.float64)
    idx = [tuple(rng.integers(0, s) for s in base.shape) for _ in range(6)]
    for ix in idx:
        p = base.copy()
        m = base.copy()
        p[ix] += h
        m[ix] -= h
        fd = (_loss(d, sc, gv, gm, **{key: p}) - _loss(d, sc, gv, gm, **{key: m})) / (2 * h)
        assert abs(fd - ana[ix]) <= 2e-3 * max(1.0, abs(fd)), (name, ix, fd, ana[ix])


def test_reference_mode_has_zero_skinned_gradients(scene):
    sc, d = scene
    gv = np.ones_like(sc["disp"])
    g = O.eg_backward(d, gv, None, sc["dT"], sc["dA"], sc["sA"], sc["disp"], full=False)
    assert not g["st"].any() and not g["sr"].any()
    assert np.abs(g["t"]).sum() > 0
