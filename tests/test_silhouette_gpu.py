"""Camera projection, projected-mesh boundary and the multi-view silhouette
loss on the GPU against the reference kernels and the FP64 oracle."""
import os

import numpy as np
import pytest
import torch

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.renderer import RendererEngine
from deepcharacters_b200.silhouette import (SilhouetteEngine, camera_projection_backward, camera_projection_forward,
                                            projected_mesh_boundary, silhouette_backward)
from oracle import oracle as O
from oracle import silhouette_oracle as SO

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference kernels (oracle/_ref) not built")
RES = 192


def _t(a, dt=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV, dt)


def nrel(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


@pytest.fixture(scope="module")
def scene():
    sc = S.render_scene(4, batch=2, views=3, width=RES, height=RES, seed=31)
    verts = _t(sc["verts"])
    v = sc["verts"].astype(np.float64)
    normals = v / np.linalg.norm(v, axis=2, keepdims=True)
    eng = RendererEngine(sc["faces"], sc["texcoords"], sc["N"], 3, RES, RES, "foregroundMask", "shadeless", 2, 2)
    face = eng.forward(verts, None, None, None, _t(sc["extr"]), _t(sc["intr"]))[1]
    dt = S.silhouette_masks(2, 3, RES, RES, seed=5, scale=RES / 512)
    crops = S.identity_crops(2, 3, RES, RES)
    return dict(sc=sc, verts=verts, normals=_t(normals.astype(np.float32)), face=face, dt=dt, crops=crops)


@needs_ref
def test_projection_matches_reference_kernels(scene):
    sc = scene["sc"]
    ex, it = _t(sc["extr"]), _t(sc["intr"])
    ref = O.RefSilhouette()
    for is_point in (1, 0):
        ours = camera_projection_forward(scene["verts"], scene["normals"], ex, it, is_point)
        theirs = ref.project(scene["verts"], scene["normals"], ex, it, is_point)
        torch.cuda.synchronize()
        assert torch.equal(ours, theirs), (is_point, nrel(ours, theirs))
    g = torch.randn((2, 3, sc["N"], 2), device=DEV, generator=torch.Generator(DEV).manual_seed(1))
    ours = camera_projection_backward(g, scene["verts"], ex, it, 1)
    theirs = ref.project_grad(g, scene["verts"], ex, it, 1)
    assert nrel(ours, theirs) < 1e-6


def test_projection_matches_fp64_oracle(scene):
    sc = scene["sc"]
    ex, it = _t(sc["extr"]), _t(sc["intr"])
    p = camera_projection_forward(scene["verts"], None, ex, it, 1)
    po = SO.project(sc["verts"], None, sc["extr"], sc["intr"], True)
    assert nrel(p, po) < 1e-6
    g = np.random.default_rng(2).normal(size=(2, 3, sc["N"], 2))
    gp = camera_projection_backward(_t(g), scene["verts"], ex, it, 1)
    assert nrel(gp, SO.project_grad(g, sc["verts"], sc["extr"], sc["intr"])) < 1e-5


def _sil_inputs(scene):
    sc = scene["sc"]
    ex, it = _t(sc["extr"]), _t(sc["intr"])
    p2d = camera_projection_forward(scene["verts"], None, ex, it, 1)
    n2d = camera_projection_forward(scene["verts"], scene["normals"], ex, it, 0)
    isb = projected_mesh_boundary(p2d, scene["face"], RES, RES)
    return p2d, n2d, isb, _t(scene["dt"], torch.uint8), _t(scene["crops"])


@needs_ref
def test_silhouette_matches_reference_kernels(scene):
    p2d, n2d, isb, dt, crops = _sil_inputs(scene)
    assert int(isb.sum()) > 0
    eng = SilhouetteEngine()
    ours = eng.forward(p2d, n2d, isb, dt, crops)
    ref = O.RefSilhouette().forward(p2d, n2d, isb, dt, crops)
    torch.cuda.synchronize()
    names = ("mv_dt_residual", "mv_dt_residual_1", "dt_image_gradient", "closest_vertex_id")
    for a, b, n in zip(ours, ref, names):
        assert torch.equal(a, b), (n, nrel(a, b))
    assert int((ours[3] >= 0).sum()) > 0
    g = torch.randn(ours[0].shape, device=DEV, generator=torch.Generator(DEV).manual_seed(3))
    g1 = torch.randn(ours[1].shape, device=DEV, generator=torch.Generator(DEV).manual_seed(4))
    gp = silhouette_backward(g, g1, ours[2], ours[3], crops)
    rgp = O.RefSilhouette().backward(g, g1, ref[2], ref[3], crops)
    assert nrel(gp, rgp) < 1e-6


def test_silhouette_matches_fp64_oracle(scene):
    p2d, n2d, isb, dt, crops = _sil_inputs(scene)
    ours = SilhouetteEngine().forward(p2d, n2d, isb, dt, crops)
    ora = SO.silhouette_forward(p2d.cpu().numpy(), n2d.cpu().numpy(), isb.cpu().numpy(), scene["dt"],
                                scene["crops"])
    assert np.array_equal(ours[3].cpu().numpy(), ora[3])
    for a, b in zip(ours[:3], ora[:3]):
        assert nrel(a, b) < 1e-6


@needs_ref
def test_mesh_boundary_matches_reference_kernels(scene):
    from deepcharacters_b200.silhouette import MeshBoundaryEngine
    sc = scene["sc"]
    ex, it = _t(sc["extr"]), _t(sc["intr"])
    eng = MeshBoundaryEngine(sc["faces"], sc["N"])
    ours = eng.forward(scene["verts"], ex, it, RES, RES)
    ref = O.ref_mesh_boundary(sc["faces"], scene["verts"], ex, it, RES, RES)
    torch.cuda.synchronize()
    assert int(ref.sum()) > 0
    assert torch.equal(ours, ref), int((ours != ref).sum())
    # from a CameraProjectionGpu result: the same points, the same flags
    p2d = camera_projection_forward(scene["verts"], None, ex, it, 1)
    assert torch.equal(eng.forward(scene["verts"], ex, it, RES, RES, points_image_space=p2d), ref)
    # a non-square raster
    ours = eng.forward(scene["verts"], ex, it, RES, RES // 2)
    ref = O.ref_mesh_boundary(sc["faces"], scene["verts"], ex, it, RES, RES // 2)
    assert torch.equal(ours, ref), int((ours != ref).sum())


def test_mesh_boundary_matches_fp64_oracle(scene):
    from deepcharacters_b200.silhouette import MeshBoundaryEngine
    sc = scene["sc"]
    ex, it = _t(sc["extr"]), _t(sc["intr"])
    ours = MeshBoundaryEngine(sc["faces"], sc["N"]).forward(scene["verts"], ex, it, RES, RES).cpu().numpy()
    p2d = SO.project(sc["verts"], None, sc["extr"], sc["intr"], True)
    ora = SO.mesh_boundary(sc["faces"], p2d, RES, RES)
    # FP64 coverage differs from FP32 only where a pixel centre sits on the
    # -0.001 / 1.001 barycentric tolerance
    assert ora.sum() > 0
    assert (ours != ora).mean() < 1e-3


def _box(P, F, x0, y0, x1, y1):
    i = len(P)
    P += [(x0, y0), (x1, y0), (x1, y1), (x0, y1)]
    F += [(i, i + 1, i + 2), (i, i + 2, i + 3)]


# sharp corners of the slivers below; at (16, 52) the pixel left of the corner
# lies in the tile before the sliver's
CORNERS = ((13, 20), (29, 40), (45, 12), (16, 52))


def test_mesh_boundary_tests_only_the_triangle_box():
    """A long sliver whose sharp vertex sits 1.1 px right of a pixel centre:
    that centre passes the widened barycentric test (-0.001 / 1.001) but lies
    outside the sliver's clamped pixel box, so the reference leaves it
    uncovered.  Three boxes cover the rest of a probe vertex's 3x3 window,
    making the probe's flag depend on that one pixel alone."""
    from deepcharacters_b200.silhouette import MeshBoundaryEngine
    W = H = 64
    P, F, probes, slivers = [], [], [], []
    for x, y in CORNERS:
        i = len(P)
        P += [(x + 0.6, y + 0.5), (x + 2000.0, y + 0.5 - 10.0), (x + 2000.0, y + 0.5 + 10.0)]
        slivers.append(len(F))
        F.append((i, i + 1, i + 2))
        _box(P, F, x - 3.0, y - 1.0, x - 1.05, y + 2.0)
        _box(P, F, x - 1.0, y - 1.0, x + 0.0, y - 0.05)
        _box(P, F, x - 1.0, y + 1.05, x + 0.0, y + 2.0)
        probes.append(len(P))
        P.append((x - 1.5, y + 0.5))
        # the pixel (x-1, y) passes the sliver's barycentric test in FP64
        a, b, c = np.array(P[i]), np.array(P[i + 1]), np.array(P[i + 2])
        pu, pv = x - 0.5, y + 0.5
        d2 = (a[1] - b[1]) * c[0] + (b[0] - a[0]) * c[1] + a[0] * b[1] - b[0] * a[1]
        d1 = (a[1] - c[1]) * b[0] + (c[0] - a[0]) * b[1] + a[0] * c[1] - c[0] * a[1]
        e2 = ((a[1] - b[1]) * pu + (b[0] - a[0]) * pv + a[0] * b[1] - b[0] * a[1]) / d2
        e1 = ((a[1] - c[1]) * pu + (c[0] - a[0]) * pv + a[0] * c[1] - c[0] * a[1]) / d1
        e = np.array([1 - e1 - e2, e1, e2])
        assert (e >= -0.001).all() and (e <= 1.001).all() and e.max() > 1.0
    p2d = np.asarray(P, np.float32)[None, None]
    faces = np.asarray(F, np.int32)
    N = p2d.shape[2]
    ora = SO.mesh_boundary(faces, p2d, W, H)
    assert all(ora[0, 0, k] == 1 for k in probes)
    eng = MeshBoundaryEngine(faces, N)
    zeros = torch.zeros((1, N, 3), device=DEV)
    ex, it = torch.zeros((1, 12), device=DEV), torch.zeros((1, 9), device=DEV)
    ours = eng.forward(zeros, ex, it, W, H, points_image_space=_t(p2d))
    assert np.array_equal(ours.cpu().numpy(), ora)
    # a hint naming the sliver at every pixel must not cover the pixel outside its box
    hint = torch.full((1, 1, H, W), -1, dtype=torch.int32, device=DEV)
    for (x, y), f in zip(CORNERS, slivers):
        hint[0, 0, y - 2:y + 3, x - 4:x + 2] = f
    hinted = eng.forward(zeros, ex, it, W, H, points_image_space=_t(p2d), face_hint=hint)
    assert np.array_equal(hinted.cpu().numpy(), ora)


def test_mesh_boundary_hint_changes_no_flag(scene):
    """The hinted coverage gives the same flags as the full one for the
    renderer's face buffer of the same views, for no hint at all (-1), and for
    random face ids (in and out of range)."""
    from deepcharacters_b200.silhouette import MeshBoundaryEngine
    sc = scene["sc"]
    ex, it = _t(sc["extr"]), _t(sc["intr"])
    eng = MeshBoundaryEngine(sc["faces"], sc["N"])
    for width, height in ((RES, RES), (RES, RES // 2)):
        full = eng.forward(scene["verts"], ex, it, width, height).clone()
        assert int(full.sum()) > 0
        g = torch.Generator(DEV).manual_seed(7)
        F = len(sc["faces"])
        hints = [torch.full((2, 3, height, width), -1, dtype=torch.int32, device=DEV),
                 torch.randint(-2, F + 5, (2, 3, height, width), generator=g, device=DEV, dtype=torch.int32)]
        if height == RES:
            hints.append(scene["face"].contiguous())
        for k, hint in enumerate(hints):
            for _ in range(2):  # two calls in a row on the same handle
                hinted = eng.forward(scene["verts"], ex, it, width, height, face_hint=hint)
                torch.cuda.synchronize()
                assert torch.equal(hinted, full), (width, height, k, int((hinted != full).sum()))


def test_fused_squared_loss_matches_the_separate_passes(scene):
    """hc_silhouette_forward_sumsq_sized gives the outputs of the plain
    forward and the loss of hc_sum_squares_loss over its residual image;
    hc_silhouette_backward_scaled_sized on (residual, 2 w) gives the adjoint
    of the plain backward on the gradient image 2 w x residual."""
    import ctypes as C
    from deepcharacters_b200 import _lib
    p2d, n2d, isb, dt, crops = _sil_inputs(scene)
    B, Cn, N = p2d.shape[0], p2d.shape[1], p2d.shape[2]
    ws = np.full(Cn, RES, np.int32)
    eng = SilhouetteEngine()
    plain = eng.forward(p2d, n2d, isb, dt, crops)
    outs = [torch.empty_like(t) for t in plain]
    acc = torch.zeros(2, dtype=torch.float64, device=DEV)
    loss = torch.zeros(2, device=DEV)
    w1 = 1e-3
    P = _lib.ptr
    _lib.call("hc_silhouette_forward_sumsq_sized", eng.handle, None, B, Cn, N, ws.ctypes.data, ws.ctypes.data,
              P(p2d), P(n2d), P(isb), P(dt), P(crops), *(P(t) for t in outs), w1, P(acc), P(loss))
    g1 = torch.empty_like(plain[1])
    _lib.call("hc_sum_squares_loss", None, g1.numel(), P(plain[1]), w1, P(acc[1:]), P(loss[1:]), P(g1))
    torch.cuda.synchronize()
    for a, b in zip(outs, plain):
        assert torch.equal(a, b)
    assert int((plain[3] >= 0).sum()) > 0 and float(loss[1]) > 0
    assert abs(float(loss[0]) - float(loss[1])) <= 1e-6 * float(loss[1])
    g = torch.randn(plain[0].shape, device=DEV, generator=torch.Generator(DEV).manual_seed(3))
    ref = silhouette_backward(g, g1, plain[2], plain[3], crops)
    out = torch.empty_like(ref)
    _lib.call("hc_silhouette_backward_scaled_sized", None, B, Cn, N, ws.ctypes.data, ws.ctypes.data, P(g),
              P(plain[1]), 2.0 * w1, P(plain[2]), P(plain[3]), P(crops), P(out))
    torch.cuda.synchronize()
    assert float(ref.abs().max()) > 0
    assert nrel(out, ref) < 1e-6  # float atomics: equal up to summation order


def test_mesh_boundary_with_an_overflowing_coverage_tile():
    """300 small triangles inside one 8x8 coverage tile: more than its bin
    holds (256 entries), so the pairs beyond it take the sweep path.  Probe
    vertices around that tile and the triangles' own vertices get the same
    flags with no hint and with a hint that names no face (every window
    left open), the reference kernels' flags, and those of the FP64 oracle up
    to pixel centres on its tolerance."""
    from deepcharacters_b200.silhouette import MeshBoundaryEngine
    W = H = 48
    rng = np.random.default_rng(17)
    P, F = [], []
    for _ in range(300):  # triangles of 1.5-3.5 px inside the pixel square [16, 24)^2
        c = rng.uniform(16.5, 23.5, 2)
        i = len(P)
        for _ in range(3):
            P.append(tuple(np.clip(c + rng.uniform(-1.75, 1.75, 2), 16.0, 24.0)))
        F.append((i, i + 1, i + 2))
    for y in range(12, 29, 2):  # probes around the tile
        for x in range(12, 29, 2):
            P.append((x + 0.25, y + 0.75))
    faces = np.asarray(F, np.int32)
    N = len(P)
    # points at z = 1000 mm seen by a camera with a 1000 px focal length land on (u, v)
    pts = np.concatenate([np.asarray(P, np.float32), np.full((N, 1), 1000.0, np.float32)], 1)[None]
    extr = np.asarray([[1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0]], np.float32)
    intr = np.asarray([[1000, 0, 0, 0, 1000, 0, 0, 0, 1]], np.float32)
    eng = MeshBoundaryEngine(faces, N)
    ours = eng.forward(_t(pts), _t(extr), _t(intr), W, H).clone()
    hint = torch.full((1, 1, H, W), -1, dtype=torch.int32, device=DEV)
    hinted = eng.forward(_t(pts), _t(extr), _t(intr), W, H, face_hint=hint)
    torch.cuda.synchronize()
    assert torch.equal(ours, hinted)
    flags = ours.cpu().numpy()
    assert 0 < int(flags.sum()) < N  # covered and open windows both occur
    if O.ref_available() and os.path.exists(O.REF_MB_LIB):
        ref = O.ref_mesh_boundary(faces, _t(pts), _t(extr), _t(intr), W, H)
        assert torch.equal(ours, ref.to(ours.device).view_as(ours))
    p2d = SO.project(pts, None, extr, intr, True)
    ora = SO.mesh_boundary(faces, p2d, W, H)
    assert int((flags != ora).sum()) <= 2  # FP64 differs only where a centre sits on the tolerance
