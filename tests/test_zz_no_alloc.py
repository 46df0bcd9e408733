"""hc_silhouette_forward_static: the silhouette forward for callers that
cannot allocate device memory (a TensorFlow op must take its memory from TF's
allocator; some hosts reserve everything at start-up).  Its scratch is a
fixed 8 MiB array inside libhc.so.  Checked through the C ABI against the
handle-based hc_silhouette_forward on two calls in a row (the array keeps
the previous call's contents, so the second call proves it is reset).

This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

from deepcharacters_b200 import _lib


def _static_call(B, C, N, U, V, ptrs, stream=None):
    return _lib.lib().hc_silhouette_forward_static(stream, B, C, N, U, V, *ptrs)


def test_rejects_calls_larger_than_the_static_scratch():
    """128 views of 1024x1024 with 40,962 points need ~23 MB of grid: refused
    before any device work (no GPU needed)."""
    dummy = [ctypes.c_void_p(16)] * 9
    st = _static_call(16, 8, 40962, 1024, 1024, dummy)
    assert st == 1
    assert b"static scratch holds 8388608 bytes" in _lib.lib().hc_last_error()


@pytest.mark.gpu
def test_static_scratch_matches_allocating_entry_point_twice():
    import torch

    from deepcharacters_b200 import synthetic as S
    from deepcharacters_b200.renderer import RendererEngine
    from deepcharacters_b200.silhouette import SilhouetteEngine, camera_projection_forward, projected_mesh_boundary

    dev = "cuda:0"
    res = 160
    t = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to(dev, dt)  # noqa: E731
    P = _lib.ptr
    eng = SilhouetteEngine()
    for call, seed in enumerate((41, 42)):
        sc = S.render_scene(3, batch=2, views=3, width=res, height=res, seed=seed)
        verts = t(sc["verts"])
        v = sc["verts"].astype(np.float64)
        normals = t((v / np.linalg.norm(v, axis=2, keepdims=True)).astype(np.float32))
        ex, it = t(sc["extr"]), t(sc["intr"])
        r = RendererEngine(sc["faces"], sc["texcoords"], sc["N"], 3, res, res, "foregroundMask", "shadeless", 2, 2)
        face = r.forward(verts, None, None, None, ex, it)[1]
        p2d = camera_projection_forward(verts, None, ex, it, 1)
        n2d = camera_projection_forward(verts, normals, ex, it, 0)
        isb = projected_mesh_boundary(p2d, face, res, res)
        dt = t(S.silhouette_masks(2, 3, res, res, seed=seed, scale=res / 512), torch.uint8)
        crops = t(S.identity_crops(2, 3, res, res))
        ref = eng.forward(p2d, n2d, isb, dt, crops)
        B, Cn, N = p2d.shape[:3]
        out = [torch.full_like(x, 7.0) for x in ref]
        st = _static_call(B, Cn, N, res, res, [P(p2d), P(n2d), P(isb), P(dt), P(crops)] + [P(x) for x in out],
                          torch.cuda.current_stream().cuda_stream)
        assert st == 0, _lib.lib().hc_last_error()
        torch.cuda.synchronize()
        assert int((ref[3] >= 0).sum()) > 0
        for a, b in zip(out, ref):
            assert torch.equal(a, b), f"call {call}"


def _need_bytes(views, N, U, V):
    """Grid scratch of one call, as documented in hc.h."""
    cells = (-(-U // 30) + 3) * (-(-V // 30) + 3)
    return 4 * (views * (3 * cells + N) + 1)


@pytest.mark.gpu
def test_static_scratch_at_its_limit():
    """8 views of 1024x1024: with 40,962 points (the documented example) and
    with the largest point count whose grid still fits the 8 MiB array (its
    last words in use), the static call equals the handle-based forward on
    synthetic points; one point more is refused with HC_ERR_INVALID."""
    import torch

    from deepcharacters_b200 import synthetic as S
    from deepcharacters_b200.silhouette import SilhouetteEngine

    dev = "cuda:0"
    B, Cn, U, V = 1, 8, 1024, 1024
    cap = 8 << 20
    n_max = (cap // 4 - 1 - B * Cn * 3 * ((-(-U // 30) + 3) * (-(-V // 30) + 3))) // (B * Cn)
    assert _need_bytes(B * Cn, n_max, U, V) <= cap < _need_bytes(B * Cn, n_max + 1, U, V)
    P = _lib.ptr
    eng = SilhouetteEngine()
    dt = torch.from_numpy(S.silhouette_masks(B, Cn, U, V, seed=5, scale=2.0)).to(dev)
    crops = torch.from_numpy(S.identity_crops(B, Cn, U, V)).to(dev)
    gen = torch.Generator(dev).manual_seed(9)
    for N in (40962, n_max):
        p2d = torch.rand((B, Cn, N, 2), device=dev, generator=gen) * torch.tensor([U, V], device=dev)
        n2d = torch.nn.functional.normalize(torch.randn((B, Cn, N, 2), device=dev, generator=gen), dim=-1)
        isb = (torch.rand((B, Cn, N), device=dev, generator=gen) < 0.05).to(torch.uint8)
        ref = eng.forward(p2d, n2d, isb, dt, crops)
        for call in range(2):
            out = [torch.full_like(x, 7.0) for x in ref]
            st = _static_call(B, Cn, N, U, V, [P(p2d), P(n2d), P(isb), P(dt), P(crops)] + [P(x) for x in out],
                              torch.cuda.current_stream().cuda_stream)
            assert st == 0, _lib.lib().hc_last_error()
            torch.cuda.synchronize()
            assert int((ref[3] >= 0).sum()) > 0
            for a, b in zip(out, ref):
                assert torch.equal(a, b), (N, call)
    N = n_max + 1
    big = [torch.zeros((B, Cn, N, 2), device=dev)] * 2 + [torch.zeros((B, Cn, N), device=dev, dtype=torch.uint8)]
    outs = [torch.zeros((B, Cn, N), device=dev), torch.zeros((B, Cn, V, U, 2), device=dev),
            torch.zeros((B, Cn, N, 2), device=dev), torch.zeros((B, Cn, V, U), device=dev)]
    st = _static_call(B, Cn, N, U, V, [P(big[0]), P(big[1]), P(big[2]), P(dt), P(crops)] + [P(x) for x in outs],
                      torch.cuda.current_stream().cuda_stream)
    assert st == 1 and b"static scratch holds 8388608 bytes" in _lib.lib().hc_last_error()
