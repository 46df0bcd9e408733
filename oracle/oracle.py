"""Python access to the test oracles -- TEST INFRASTRUCTURE ONLY.

* ``libhcoracle.so``: the CPU restatement of the reference path (FP64 and
  FP32 variants), built by ``make -C oracle``.
* ``_ref/libhcref.so``: the reference's own CUDA kernels, compiled unmodified
  from the reference tree with the harness in ``oracle/ref`` (``make -C
  oracle ref``); needs a GPU.

Only tests/, the smoke check and bench.py's CPU-baseline / reference legs
import this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "libhcoracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libhcref.so")

ALBEDO = {"vertexColor": 0, "textured": 1, "normal": 2, "lighting": 3, "foregroundMask": 4, "position": 5,
          "depth": 6, "uv": 7}
SHADING = {"shaded": 0, "shadeless": 1}

_olib = None
_rlib = None


def oracle_lib() -> C.CDLL:
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            raise RuntimeError(f"{ORACLE_LIB} missing: run `make -C oracle`")
        _olib = C.CDLL(ORACLE_LIB)
        for name in ("hco_render_forward_f64", "hco_render_forward_f32"):
            getattr(_olib, name).restype = C.c_int
    return _olib


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib() -> C.CDLL:
    global _rlib
    if _rlib is None:
        if not os.path.exists(REF_LIB):
            raise RuntimeError(f"{REF_LIB} missing: run `make -C oracle ref` where the reference tree exists")
        _rlib = C.CDLL(REF_LIB)
        _rlib.hcref_renderer_create.restype = C.c_void_p
        _rlib.hcref_renderer_create.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                                C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        _rlib.hcref_renderer_destroy.argtypes = [C.c_void_p]
        _rlib.hcref_render_forward.restype = C.c_int
        _rlib.hcref_render_forward.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 3 + [C.c_int, C.c_int] + \
            [C.c_void_p] * 3 + [C.c_void_p] * 7 + [C.c_int]
        _rlib.hcref_render_backward.restype = C.c_int
        _rlib.hcref_render_backward.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 4 + [C.c_int, C.c_int] + \
            [C.c_void_p] * 12
    return _rlib


def _p(a):
    if a is None:
        return None
    return a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr()


def _c(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


def render_forward(faces, texcoords, B, C_, W, H, albedo, shading, verts, colors, texture, sh, extr, intr,
                   precision="f64", nthreads=0, fragile=True):
    """CPU oracle forward.  Returns a dict of numpy arrays."""
    faces = _c(faces, np.int32).reshape(-1)
    F = faces.size // 3
    verts = _c(verts, np.float32)
    N = verts.reshape(B, -1, 3).shape[1]
    colors = _c(colors, np.float32)
    texture = _c(texture, np.float32)
    TH, TW = (texture.shape[1], texture.shape[2]) if texture is not None and texture.ndim == 4 else (0, 0)
    tc = _c(texcoords, np.float32) if texcoords is not None else np.zeros(6 * F, np.float32)
    sh = _c(sh, np.float32) if sh is not None else np.zeros((B, C_, 27), np.float32)
    extr = _c(extr, np.float32)
    intr = _c(intr, np.float32)
    out = {
        "bary": np.zeros((B, C_, H, W, 2), np.float32),
        "face": np.zeros((B, C_, H, W), np.int32),
        "render": np.zeros((B, C_, H, W, 3), np.float32),
        "vnormal": np.zeros((B, C_, N, 3), np.float32),
        "depth_q": np.zeros((B, C_, H, W), np.int32),
        "tie_count": np.zeros((B, C_, H, W), np.int32),
        "fragile": np.zeros((B, C_, H, W), np.uint8),
    }
    fn = getattr(oracle_lib(), f"hco_render_forward_{precision}")
    st = fn(C.c_int(N), C.c_int(F), C.c_void_p(_p(faces)), C.c_void_p(_p(tc)), C.c_int(B), C.c_int(C_),
            C.c_int(W), C.c_int(H), C.c_int(ALBEDO[albedo]), C.c_int(SHADING[shading]), C.c_void_p(_p(verts)),
            C.c_void_p(_p(colors)), C.c_void_p(_p(texture)), C.c_int(TH), C.c_int(TW), C.c_void_p(_p(sh)),
            C.c_void_p(_p(extr)), C.c_void_p(_p(intr)), C.c_void_p(_p(out["bary"])), C.c_void_p(_p(out["face"])),
            C.c_void_p(_p(out["render"])), C.c_void_p(_p(out["vnormal"])), C.c_void_p(_p(out["depth_q"])),
            C.c_void_p(_p(out["tie_count"])), C.c_void_p(_p(out["fragile"]) if fragile else None),
            C.c_int(nthreads))
    if st != 0:
        raise RuntimeError("oracle render failed")
    return out


class RefRenderer:
    """The reference rasterizer kernels (GPU), driven per frame like the TF op."""

    def __init__(self, faces, texcoords, N, C_, W, H, albedo, shading, normal_mode="none", image_filter_size=2,
                 texture_filter_size=2):
        L = ref_lib()
        f = _c(faces, np.int32).reshape(-1)
        tc = None if texcoords is None else _c(texcoords, np.float32)
        nm = {"normal": 0, "position": 1, "none": 2, "face": 3}[normal_mode]
        # the op forces shadeless for modes other than vertexColor/textured
        sm = SHADING[shading] if albedo in ("vertexColor", "textured") else 1
        self.N, self.C, self.W, self.H = N, C_, W, H
        self._f, self._tc = f, tc
        self.h = L.hcref_renderer_create(N, _p(f), f.size // 3, _p(tc), C_, W, H, ALBEDO[albedo], sm, nm,
                                         image_filter_size, texture_filter_size)

    def __del__(self):
        if getattr(self, "h", None) and _rlib is not None:
            _rlib.hcref_renderer_destroy(self.h)
            self.h = None

    def forward(self, B, verts, colors, texture, sh, extr, intr, depth=True, inverses=False, sync_each=1):
        """torch CUDA tensors in; returns dict of torch tensors."""
        import torch
        dev = verts.device
        TH, TW = (texture.shape[1], texture.shape[2]) if texture is not None else (0, 0)
        o = {
            "bary": torch.zeros((B, self.C, self.H, self.W, 2), device=dev),
            "face": torch.zeros((B, self.C, self.H, self.W), device=dev, dtype=torch.int32),
            "render": torch.zeros((B, self.C, self.H, self.W, 3), device=dev),
            "vnormal": torch.zeros((B, self.C, self.N, 3), device=dev),
            "depth_q": torch.zeros((B, self.C, self.H, self.W), device=dev, dtype=torch.int32) if depth else None,
            "inv": torch.zeros((B, self.C, 32), device=dev) if inverses else None,
        }
        torch.cuda.synchronize()
        st = ref_lib().hcref_render_forward(self.h, B, _p(verts), _p(colors), _p(texture), TH, TW, _p(sh), _p(extr),
                                            _p(intr), _p(o["bary"]), _p(o["face"]), _p(o["render"]),
                                            _p(o["vnormal"]), None, _p(o["depth_q"]), _p(o["inv"]), sync_each)
        if st != 0:
            raise RuntimeError(f"reference forward failed: cuda error {st}")
        return o

    def backward(self, B, render_grad, verts, colors, texture, sh, target, vnormal, bary, face, extr, intr):
        import torch
        dev = verts.device
        TH, TW = texture.shape[1], texture.shape[2]
        o = {
            "vertex_pos_grad": torch.zeros((B, self.N, 3), device=dev),
            "vertex_color_grad": torch.zeros((B, self.N, 3), device=dev),
            "texture_grad": torch.zeros((B, TH, TW, 3), device=dev),
            "sh_coeff_grad": torch.zeros((B, self.C, 27), device=dev),
        }
        torch.cuda.synchronize()
        st = ref_lib().hcref_render_backward(self.h, B, _p(render_grad), _p(verts), _p(colors), _p(texture), TH, TW,
                                             _p(sh), _p(target), _p(vnormal), _p(bary), _p(face), _p(extr), _p(intr),
                                             _p(o["vertex_pos_grad"]), _p(o["vertex_color_grad"]),
                                             _p(o["texture_grad"]), _p(o["sh_coeff_grad"]))
        if st != 0:
            raise RuntimeError(f"reference backward failed: cuda error {st}")
        return o
