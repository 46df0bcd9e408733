"""Edge cases of the raster, the mesh boundary and the silhouette loss
against the reference kernels: a mesh behind the camera, a mesh half out of
the frame (negative pixel coordinates), degenerate triangles, odd raster
sizes with every tile size, and no boundary at all."""
import numpy as np
import pytest
import torch

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.silhouette import MeshBoundaryEngine, SilhouetteEngine, camera_projection_forward
from oracle import oracle as O

from test_renderer_gpu import run_ours, run_ref  # noqa: E402 (same directory)

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not O.ref_available(), reason="reference kernels not built")]
DEV = "cuda:0"


def _t(a, dt=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV, dt)


def _match(sc, albedo="vertexColor", shading="shaded", tile=16, cap=512):
    ours = run_ours(sc, albedo, shading, tile, cap)
    ref = run_ref(sc, albedo, shading)
    tie = ours["tie_count"] >= 2
    assert not (ours["face"] != ref["face"])[~tie].any()
    same = (ours["face"] == ref["face"]) & (ref["face"] >= 0) & ~tie
    assert np.array_equal(ours["bary"][same], ref["bary"][same])
    np.testing.assert_allclose(ours["render"][same], ref["render"][same], rtol=1e-5, atol=1e-5)
    bg = ref["face"] < 0
    assert np.all(ours["render"][bg] == 0) and np.all(ours["bary"][bg] == 0)
    return ours, ref


def _cam_centre(extr12):
    E = np.asarray(extr12, np.float64).reshape(3, 4)
    return -E[:, :3].T @ E[:, 3]


def test_mesh_behind_the_camera_renders_nothing():
    sc = S.render_scene(3, batch=1, views=1, width=64, height=48, seed=3)
    c = _cam_centre(sc["extr"][0, :12])
    sc["verts"] = (sc["verts"] + 2.0 * c).astype(np.float32)  # well behind the camera
    ours, ref = _match(sc)
    assert (ref["face"] < 0).all() and (ours["face"] < 0).all()


@pytest.mark.parametrize("tile", [8, 16, 32])
def test_mesh_half_out_of_the_frame(tile):
    sc = S.render_scene(3, batch=2, views=2, width=80, height=60, seed=5)
    # +1300 mm in y: the upper part projects above the image (negative v)
    sc["verts"] = (sc["verts"] + np.array([0.0, 1300.0, 0.0], np.float32)).astype(np.float32)
    ours, ref = _match(sc, tile=tile)
    cov = ref["face"] >= 0
    assert 0 < cov.mean() < 0.5


def test_degenerate_triangles():
    sc = S.render_scene(3, batch=1, views=2, width=72, height=56, seed=7)
    f = sc["faces"]
    # repeated-vertex and collinear triangles next to the real ones
    deg = np.stack([f[:40, 0], f[:40, 0], f[:40, 1]], 1)
    col = np.stack([f[40:60, 0], f[40:60, 1], f[40:60, 1]], 1)
    sc["faces"] = np.concatenate([f, deg, col]).astype(np.int32)
    tc = np.asarray(sc["texcoords"], np.float32).reshape(-1, 6)
    sc["texcoords"] = np.concatenate([tc, tc[:60]]).reshape(-1).astype(np.float32)
    sc["F"] = sc["faces"].shape[0]
    _match(sc)


@pytest.mark.parametrize("size,tile", [((37, 23), 8), ((37, 23), 16), ((37, 23), 32), ((3, 5), 8)])
def test_odd_raster_sizes(size, tile):
    W, H = size
    sc = S.render_scene(2, batch=1, views=2, width=W, height=H, seed=9)
    ours, ref = _match(sc, tile=tile)
    assert (ref["face"] >= 0).any()


def test_boundary_and_silhouette_without_visible_points():
    sc = S.render_scene(2, batch=1, views=2, width=48, height=48, seed=11)
    verts = _t(sc["verts"] + np.array([1.0e5, 0.0, 0.0], np.float32))  # every point far off-screen
    ex, it = _t(sc["extr"]), _t(sc["intr"])
    eng = MeshBoundaryEngine(sc["faces"], sc["N"])
    ours = eng.forward(verts, ex, it, 48, 48)
    ref = O.ref_mesh_boundary(sc["faces"], verts, ex, it, 48, 48)
    torch.cuda.synchronize()
    assert torch.equal(ours, ref) and int(ours.sum()) == 0
    p2d = camera_projection_forward(verts, None, ex, it, 1)
    dt = _t(S.silhouette_masks(1, 2, 48, 48, seed=2, scale=48 / 512), torch.uint8)
    crops = _t(S.identity_crops(1, 2, 48, 48))
    isb = torch.zeros((1, 2, sc["N"]), dtype=torch.uint8, device=DEV)
    a = SilhouetteEngine().forward(p2d, p2d, isb, dt, crops)
    b = O.RefSilhouette().forward(p2d, p2d, isb, dt, crops)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    assert int((a[3] >= 0).sum()) == 0
