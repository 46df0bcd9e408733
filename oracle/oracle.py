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
        for name in ("hco_render_forward_f64", "hco_render_forward_f32", "hco_render_backward_f64",
                     "hco_render_backward_f32", "hco_eg_forward_f64", "hco_eg_forward_f32", "hco_eg_backward_f64",
                     "hco_eg_backward_f32", "hco_eg_forward_f64d"):
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
            [C.c_void_p] * 11
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


def render_backward(faces, texcoords, B, C_, W, H, albedo, shading, grad, verts, colors, texture, sh, target,
                    vnormal, bary, face, extr, intr, ifs=2, tfs=2, precision="f64", nthreads=0):
    """CPU oracle adjoint.  Returns dict of numpy gradient arrays."""
    faces = _c(faces, np.int32).reshape(-1)
    F = faces.size // 3
    verts = _c(verts, np.float32)
    N = verts.reshape(B, -1, 3).shape[1]
    texture = _c(texture, np.float32)
    TH, TW = (texture.shape[1], texture.shape[2]) if texture is not None and texture.ndim == 4 else (0, 0)
    tc = _c(texcoords, np.float32) if texcoords is not None else np.zeros(6 * F, np.float32)
    arrs = [_c(a, np.float32) for a in (grad, colors, sh, target, vnormal, bary, extr, intr)]
    grad, colors, sh, target, vnormal, bary, extr, intr = arrs
    face = _c(face, np.int32)
    out = {"vertex_pos_grad": np.zeros((B, N, 3), np.float32), "vertex_color_grad": np.zeros((B, N, 3), np.float32),
           "texture_grad": np.zeros((B, max(TH, 1), max(TW, 1), 3), np.float32),
           "sh_coeff_grad": np.zeros((B, C_, 27), np.float32)}
    fn = getattr(oracle_lib(), f"hco_render_backward_{precision}")
    vp_ = C.c_void_p
    st = fn(C.c_int(N), C.c_int(F), vp_(_p(faces)), vp_(_p(tc)), C.c_int(B), C.c_int(C_), C.c_int(W), C.c_int(H),
            C.c_int(ALBEDO[albedo]), C.c_int(SHADING[shading]), C.c_int(ifs), C.c_int(tfs), vp_(_p(grad)),
            vp_(_p(verts)), vp_(_p(colors)), vp_(_p(texture)), C.c_int(TH), C.c_int(TW), vp_(_p(sh)),
            vp_(_p(target)), vp_(_p(vnormal)), vp_(_p(bary)), vp_(_p(face)), vp_(_p(extr)), vp_(_p(intr)),
            vp_(_p(out["vertex_pos_grad"])), vp_(_p(out["vertex_color_grad"])),
            vp_(_p(out["texture_grad"]) if TH > 0 else None), vp_(_p(out["sh_coeff_grad"])), C.c_int(nthreads))
    if st != 0:
        raise RuntimeError("oracle render backward failed")
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


# ---------------------------------------------------------------------------
# embedded graph
# ---------------------------------------------------------------------------
def _eg_arrays(d):
    i32 = lambda a: _c(a, np.int32)  # noqa: E731
    f32 = lambda a: _c(a, np.float32)  # noqa: E731
    return dict(base=f32(d.base_vertices), faces=i32(d.faces), nv=i32(d.node_vertex), v2n_off=i32(d.v2n_offsets),
                v2n_size=i32(d.v2n_sizes), v2n_idx=i32(d.v2n_indices), v2n_w=f32(d.v2n_weights),
                n2v_off=i32(d.n2v_offsets), n2v_size=i32(d.n2v_sizes), n2v_idx=i32(d.n2v_indices),
                n2v_w=f32(d.n2v_weights),
                markers=f32(d.markers) if d.markers is not None else np.zeros((1, 3), np.float32),
                m2n=i32(d.marker_node) if d.marker_node is not None else np.zeros(1, np.int32),
                Mk=0 if d.markers is None else len(d.markers))


def eg_forward(d, dT, dA, sT, sA, disp, precision="f64"):
    """CPU oracle EG forward; d is an EGData.  numpy in / out."""
    a = _eg_arrays(d)
    B = dT.shape[0]
    N, M, F, Mk = a["base"].shape[0], a["nv"].shape[0], a["faces"].size // 3, a["Mk"]
    ins = [_c(x, np.float32) for x in (dT, dA, sT, sA, disp)]
    odt = np.float64 if precision == "f64d" else np.float32
    out = {"vertices": np.zeros((B, N, 3), odt), "normals": np.zeros((B, N, 3), odt),
           "markers": np.zeros((B, max(Mk, 1), 3), odt), "graph": np.zeros((B, M, 3), odt)}
    fn = getattr(oracle_lib(), f"hco_eg_forward_{precision}")
    vp_ = C.c_void_p
    st = fn(B, N, M, Mk, F, vp_(_p(a["base"])), vp_(_p(a["faces"])), vp_(_p(a["nv"])), vp_(_p(a["v2n_off"])),
            vp_(_p(a["v2n_size"])), vp_(_p(a["v2n_idx"])), vp_(_p(a["v2n_w"])), vp_(_p(a["markers"])),
            vp_(_p(a["m2n"])), *(vp_(_p(x)) for x in ins), vp_(_p(out["vertices"])), vp_(_p(out["normals"])),
            vp_(_p(out["markers"])), vp_(_p(out["graph"])))
    if st != 0:
        raise RuntimeError("oracle eg forward failed")
    return out


def eg_backward(d, gv, gm, dT, dA, sA, disp, full=False, precision="f64"):
    a = _eg_arrays(d)
    B = gv.shape[0]
    N, M, Mk = a["base"].shape[0], a["nv"].shape[0], a["Mk"]
    n2m = np.full(M, -1, np.int32)
    if Mk:
        n2m[a["m2n"]] = np.arange(Mk, dtype=np.int32)
    gv, dT, dA, sA, disp = (_c(x, np.float32) for x in (gv, dT, dA, sA, disp))
    gm = _c(gm, np.float32) if (gm is not None and Mk) else None
    out = {k: np.zeros((B, M, 3), np.float32) for k in ("t", "r", "st", "sr")}
    out["disp"] = np.zeros((B, N, 3), np.float32)
    fn = getattr(oracle_lib(), f"hco_eg_backward_{precision}")
    vp_ = C.c_void_p
    st = fn(B, N, M, Mk, vp_(_p(a["base"])), vp_(_p(a["nv"])), vp_(_p(a["v2n_off"])), vp_(_p(a["v2n_size"])),
            vp_(_p(a["v2n_idx"])), vp_(_p(a["v2n_w"])), vp_(_p(a["n2v_off"])), vp_(_p(a["n2v_size"])),
            vp_(_p(a["n2v_idx"])), vp_(_p(a["n2v_w"])), vp_(_p(n2m)), vp_(_p(a["markers"])), vp_(_p(gv)),
            vp_(_p(gm)), vp_(_p(dT)), vp_(_p(dA)), vp_(_p(sA)), vp_(_p(disp)), int(full), vp_(_p(out["t"])),
            vp_(_p(out["r"])), vp_(_p(out["st"])), vp_(_p(out["sr"])), vp_(_p(out["disp"])))
    if st != 0:
        raise RuntimeError("oracle eg backward failed")
    return out


class RefArap:
    """The reference ARAP regulariser kernels (GPU), on torch CUDA tensors
    (EmbeddedGraphArapGPUOp.cu:10-97, EmbeddedGraphArapGPUOpGrad.cu:9-104)."""

    def __init__(self, base, node_vertex, off, size, idx, rigid, maxc, device):
        import torch
        t = lambda x, dt: torch.from_numpy(np.ascontiguousarray(np.asarray(x, dt))).to(device)  # noqa: E731
        self.d = {"base": t(base, np.float32), "nv": t(node_vertex, np.int32), "off": t(off, np.int32),
                  "size": t(size, np.int32), "idx": t(idx, np.int32), "rigid": t(rigid, np.float32)}
        self.M, self.maxc = len(node_vertex), int(maxc)
        L = ref_lib()
        L.hcref_arap_forward.restype = C.c_int
        L.hcref_arap_forward.argtypes = [C.c_int] * 3 + [C.c_void_p] * 11
        L.hcref_arap_backward.restype = C.c_int
        L.hcref_arap_backward.argtypes = [C.c_int] * 3 + [C.c_void_p] * 10

    def forward(self, T, A):
        import torch
        B, dev, d = T.shape[0], T.device, self.d
        loss = torch.zeros((B, self.M, self.maxc, 3), device=dev)
        w = torch.zeros((B, self.M, self.maxc), device=dev)
        rot = torch.zeros((B, self.M, 3), device=dev)
        torch.cuda.synchronize()
        st = ref_lib().hcref_arap_forward(B, self.M, self.maxc, _p(d["size"]), _p(d["idx"]), _p(d["off"]),
                                          _p(d["rigid"]), _p(d["nv"]), _p(d["base"]), _p(T), _p(A), _p(loss), _p(w),
                                          _p(rot))
        assert st == 0, st
        return loss, w, rot

    def backward(self, gloss, A):
        import torch
        B, dev, d = A.shape[0], A.device, self.d
        gT = torch.zeros((B, self.M, 3), device=dev)
        gA = torch.zeros((B, self.M, 3), device=dev)
        torch.cuda.synchronize()
        st = ref_lib().hcref_arap_backward(B, self.M, self.maxc, _p(d["size"]), _p(d["idx"]), _p(d["off"]),
                                           _p(d["rigid"]), _p(d["nv"]), _p(d["base"]), _p(gloss), _p(A), _p(gT),
                                           _p(gA))
        assert st == 0, st
        return gT, gA


class RefEG:
    """The reference embedded-graph kernels (GPU), on torch CUDA tensors."""

    def __init__(self, d, device):
        import torch
        a = _eg_arrays(d)
        self.N, self.M, self.F, self.Mk = a["base"].shape[0], a["nv"].shape[0], a["faces"].size // 3, a["Mk"]
        # vertex -> face lists in the reference's order
        faces = a["faces"].reshape(-1, 3)
        lists = [[] for _ in range(self.N)]
        for f, (x, y, z) in enumerate(faces):
            for v in dict.fromkeys((int(x), int(y), int(z))):
                lists[v].append(f)
        vf = np.array([f for L in lists for f in L], np.int32)
        starts = np.cumsum([0] + [len(L) for L in lists[:-1]]).astype(np.int32)
        vfid = np.stack([starts, np.array([len(L) for L in lists], np.int32)], 1)
        n2m = np.full(self.M, -1, np.int32)
        if self.Mk:
            n2m[a["m2n"]] = np.arange(self.Mk, dtype=np.int32)
        t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(device)  # noqa: E731
        self.d = {k: t(v) for k, v in a.items() if k != "Mk"}
        self.d["vf"], self.d["vfid"], self.d["n2m"] = t(vf), t(vfid), t(n2m)
        L = ref_lib()
        L.hcref_eg_forward.restype = C.c_int
        L.hcref_eg_forward.argtypes = [C.c_int] * 5 + [C.c_void_p] * 22
        L.hcref_eg_backward.restype = C.c_int
        L.hcref_eg_backward.argtypes = [C.c_int] * 4 + [C.c_void_p] * 21

    def forward(self, dT, dA, sT, sA, disp):
        import torch
        B, dev = dT.shape[0], dT.device
        o = {"vertices": torch.zeros((B, self.N, 3), device=dev), "normals": torch.zeros((B, self.N, 3), device=dev),
             "markers": torch.zeros((B, max(self.Mk, 1), 3), device=dev),
             "graph": torch.zeros((B, self.M, 3), device=dev), "da": torch.zeros((B, self.M, 3), device=dev),
             "sa": torch.zeros((B, self.M, 3), device=dev)}
        d = self.d
        torch.cuda.synchronize()
        st = ref_lib().hcref_eg_forward(B, self.N, self.M, self.Mk, self.F, _p(d["base"]), _p(d["faces"]), _p(d["vf"]),
                                        _p(d["vfid"]), _p(d["nv"]), _p(d["v2n_off"]), _p(d["v2n_size"]),
                                        _p(d["v2n_idx"]), _p(d["v2n_w"]), _p(d["m2n"]), _p(d["markers"]), _p(dT),
                                        _p(dA), _p(sT), _p(sA), _p(disp), _p(o["vertices"]), _p(o["normals"]),
                                        _p(o["markers"]), _p(o["graph"]), _p(o["da"]), _p(o["sa"]))
        if st != 0:
            raise RuntimeError(f"reference eg forward failed: {st}")
        return o

    def backward(self, gv, gm, dA, sA):
        import torch
        B, dev = gv.shape[0], gv.device
        o = {k: torch.zeros((B, self.M, 3), device=dev) for k in ("t", "r", "st", "sr")}
        o["disp"] = torch.zeros((B, self.N, 3), device=dev)
        d = self.d
        torch.cuda.synchronize()
        st = ref_lib().hcref_eg_backward(B, self.N, self.M, self.Mk, _p(d["base"]), _p(d["nv"]), _p(d["v2n_off"]),
                                         _p(d["v2n_size"]), _p(d["v2n_idx"]), _p(d["v2n_w"]), _p(d["n2v_off"]),
                                         _p(d["n2v_size"]), _p(d["n2v_idx"]), _p(d["n2v_w"]), _p(d["n2m"]),
                                         _p(d["markers"]), _p(gv), _p(gm), _p(dA), _p(sA), _p(o["t"]), _p(o["r"]),
                                         _p(o["st"]), _p(o["sr"]), _p(o["disp"]))
        if st != 0:
            raise RuntimeError(f"reference eg backward failed: {st}")
        return o


# ---------------------------------------------------------------------------
# skinning (reference GPU kernels, fed with given dual quaternions / transforms)
# ---------------------------------------------------------------------------
class RefSkin:
    def __init__(self, ch):
        L = ref_lib()
        L.hcref_dq_forward.restype = C.c_int
        L.hcref_dq_forward.argtypes = [C.c_int] * 6 + [C.c_void_p] * 9
        L.hcref_dq_backward.restype = C.c_int
        L.hcref_dq_backward.argtypes = [C.c_int] * 6 + [C.c_void_p] * 16
        L.hcref_lbs_forward.restype = C.c_int
        L.hcref_lbs_forward.argtypes = [C.c_int] * 6 + [C.c_void_p] * 10
        L.hcref_lbs_backward.restype = C.c_int
        L.hcref_lbs_backward.argtypes = [C.c_int] * 6 + [C.c_void_p] * 17
        self.ch = ch
        i32 = lambda a: np.ascontiguousarray(a, np.int32)  # noqa: E731
        f32 = lambda a: np.ascontiguousarray(a, np.float32)  # noqa: E731
        self.h = dict(parent=i32(ch.parent), type=i32(ch.joint_type), doff=i32(ch.dof_offsets), dj=i32(ch.dof_joint),
                      sj=i32(ch.skin_joint), si=i32(ch.skin_index), bv=f32(ch.base_vertices),
                      bn=f32(ch.base_normals))
        self.N, self.K = ch.skin_index.shape
        self.S, self.J, self.D = ch.n_skin, ch.n_joints, ch.n_dofs

    def dq_forward(self, dq, weights):
        import torch
        B, dev = dq.shape[0], dq.device
        o = [torch.zeros((B, self.N, 3), device=dev), torch.zeros((B, self.N, 3), device=dev),
             torch.zeros((B, self.S, 8), device=dev), torch.zeros((B, self.N, self.K), device=dev)]
        torch.cuda.synchronize()
        h = self.h
        st = ref_lib().hcref_dq_forward(B, self.N, self.S, self.K, self.J, self.D, _p(h["si"]), _p(h["bv"]),
                                        _p(h["bn"]), _p(weights), _p(dq), *(_p(t) for t in o))
        if st != 0:
            raise RuntimeError(f"reference dq forward failed: {st}")
        return o

    def dq_backward(self, gv, vpos, gpos, gaxis, dq, weights, file_weights):
        import torch
        B, dev = gv.shape[0], gv.device
        gd = torch.zeros((B, self.D), device=dev)
        gw = torch.zeros((B, self.N, self.K), device=dev)
        fw = np.ascontiguousarray(file_weights, np.float32)
        h = self.h
        torch.cuda.synchronize()
        st = ref_lib().hcref_dq_backward(B, self.N, self.S, self.K, self.J, self.D, _p(h["parent"]), _p(h["type"]),
                                         _p(h["doff"]), _p(h["dj"]), _p(h["sj"]), _p(h["si"]), _p(fw), _p(h["bv"]),
                                         _p(gv), _p(vpos), _p(gpos), _p(gaxis), _p(dq), _p(weights), _p(gd), _p(gw))
        if st != 0:
            raise RuntimeError(f"reference dq backward failed: {st}")
        return gd, gw

    def lbs_forward(self, xf12_host, weights, disp):
        import torch
        B, dev = weights.shape[0], weights.device
        o = [torch.zeros((B, self.N, 3), device=dev), torch.zeros((B, self.N, 3), device=dev),
             torch.zeros((B, self.S, 12), device=dev), torch.zeros((B, self.N, self.K), device=dev)]
        xf = np.ascontiguousarray(xf12_host, np.float32)
        h = self.h
        torch.cuda.synchronize()
        st = ref_lib().hcref_lbs_forward(B, self.N, self.S, self.K, self.J, self.D, _p(h["si"]), _p(h["bv"]),
                                         _p(h["bn"]), _p(weights), _p(disp), _p(xf), *(_p(t) for t in o))
        if st != 0:
            raise RuntimeError(f"reference lbs forward failed: {st}")
        return o

    def lbs_backward(self, gv, vpos, gpos, gaxis, xf12_dev, weights, file_weights):
        import torch
        B, dev = gv.shape[0], gv.device
        gd = torch.zeros((B, self.D), device=dev)
        gw = torch.zeros((B, self.N, self.K), device=dev)
        gdisp = torch.zeros((B, self.N, 3), device=dev)
        fw = np.ascontiguousarray(file_weights, np.float32)
        h = self.h
        torch.cuda.synchronize()
        st = ref_lib().hcref_lbs_backward(B, self.N, self.S, self.K, self.J, self.D, _p(h["parent"]), _p(h["type"]),
                                          _p(h["doff"]), _p(h["dj"]), _p(h["sj"]), _p(h["si"]), _p(fw), _p(h["bv"]),
                                          _p(gv), _p(vpos), _p(gpos), _p(gaxis), _p(xf12_dev), _p(weights), _p(gd),
                                          _p(gw), _p(gdisp))
        if st != 0:
            raise RuntimeError(f"reference lbs backward failed: {st}")
        return gd, gw, gdisp


# ---------------------------------------------------------------------------
# camera projection / silhouette (reference GPU kernels)
# ---------------------------------------------------------------------------
class RefSilhouette:
    def __init__(self):
        L = ref_lib()
        L.hcref_projection_forward.restype = C.c_int
        L.hcref_projection_forward.argtypes = [C.c_int] * 3 + [C.c_void_p] * 4 + [C.c_int, C.c_void_p]
        L.hcref_projection_backward.restype = C.c_int
        L.hcref_projection_backward.argtypes = [C.c_int] * 3 + [C.c_void_p] * 4 + [C.c_int, C.c_void_p]
        L.hcref_silhouette_forward.restype = C.c_int
        L.hcref_silhouette_forward.argtypes = [C.c_int] * 5 + [C.c_void_p] * 9
        L.hcref_silhouette_backward.restype = C.c_int
        L.hcref_silhouette_backward.argtypes = [C.c_int] * 5 + [C.c_void_p] * 6

    def project(self, pts, vecs, extr, intr, is_point):
        import torch
        B, N = pts.shape[:2]
        Cn = extr.reshape(B, -1).shape[1] // 12
        out = torch.zeros((B, Cn, N, 2), device=pts.device)
        torch.cuda.synchronize()
        st = ref_lib().hcref_projection_forward(B, Cn, N, _p(pts), _p(vecs), _p(extr), _p(intr), int(is_point),
                                                _p(out))
        if st != 0:
            raise RuntimeError(f"reference projection failed: {st}")
        return out

    def project_grad(self, g, pts, extr, intr, is_point):
        import torch
        B, Cn, N = g.shape[:3]
        out = torch.zeros((B, N, 3), device=g.device)
        torch.cuda.synchronize()
        st = ref_lib().hcref_projection_backward(B, Cn, N, _p(g), _p(pts), _p(extr), _p(intr), int(is_point), _p(out))
        if st != 0:
            raise RuntimeError(f"reference projection grad failed: {st}")
        return out

    def forward(self, p2d, n2d, isb, dt, crops):
        import torch
        B, Cn, N = p2d.shape[:3]
        U, V = dt.shape[2], dt.shape[3]
        dev = p2d.device
        o = [torch.zeros((B, Cn, N), device=dev), torch.zeros((B, Cn, V, U, 2), device=dev),
             torch.zeros((B, Cn, N, 2), device=dev), torch.zeros((B, Cn, V, U), device=dev)]
        torch.cuda.synchronize()
        st = ref_lib().hcref_silhouette_forward(B, Cn, N, U, V, _p(p2d), _p(n2d), _p(isb), _p(dt), _p(crops),
                                                *(_p(t) for t in o))
        if st != 0:
            raise RuntimeError(f"reference silhouette failed: {st}")
        return o

    def backward(self, g, g1, dtg, closest, crops):
        import torch
        B, Cn, N = g.shape
        V, U = closest.shape[2], closest.shape[3]
        out = torch.zeros((B, Cn, N, 2), device=g.device)
        torch.cuda.synchronize()
        st = ref_lib().hcref_silhouette_backward(B, Cn, N, U, V, _p(g), _p(g1), _p(dtg), _p(closest), _p(crops),
                                                 _p(out))
        if st != 0:
            raise RuntimeError(f"reference silhouette grad failed: {st}")
        return out


# ---------------------------------------------------------------------------
# projected-mesh boundary (reference GPU kernels, separate library)
# ---------------------------------------------------------------------------
REF_MB_LIB = os.path.join(HERE, "_ref", "libhcref_mb.so")
_mblib = None


def ref_mesh_boundary(faces, pts, extr, intr, width, height):
    """ProjectedMeshBoundaryGpu through the reference's own kernels
    (Skeletool/Mesh/CUDABasedRasterization.cu): bool [B,C,N] as uint8."""
    import torch
    global _mblib
    if _mblib is None:
        if not os.path.exists(REF_MB_LIB):
            raise RuntimeError(f"{REF_MB_LIB} missing: run `make -C oracle ref` where the reference tree exists")
        _mblib = C.CDLL(REF_MB_LIB)
        _mblib.hcref_mesh_boundary.restype = C.c_int
        _mblib.hcref_mesh_boundary.argtypes = [C.c_int] * 6 + [C.c_void_p] * 5
    B, N = pts.shape[:2]
    Cn = extr.reshape(B, -1).shape[1] // 12
    f = torch.as_tensor(np.ascontiguousarray(faces, np.int32)).to(pts.device)
    out = torch.zeros((B, Cn, N), device=pts.device, dtype=torch.uint8)
    torch.cuda.synchronize()
    st = _mblib.hcref_mesh_boundary(B, Cn, N, f.shape[0], int(width), int(height), _p(f), _p(pts), _p(extr),
                                    _p(intr), _p(out))
    if st != 0:
        raise RuntimeError(f"reference mesh boundary failed: {st}")
    return out


# ---------------------------------------------------------------------------
# UV-space maps (reference host class + kernels)
# ---------------------------------------------------------------------------
class RefUV:
    """The reference renderer object in a compute_normal_map mode
    (CUDABasedRasterization.cpp, host texel table built on the first call)."""

    def __init__(self, faces, texcoords, N, C_, W, H, normal_mode, albedo="vertexColor", shading="shadeless"):
        L = ref_lib()
        L.hcref_uv_create.restype = C.c_void_p
        L.hcref_uv_create.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                      C.c_char_p, C.c_char_p, C.c_char_p]
        L.hcref_uv_forward.restype = C.c_int
        L.hcref_uv_forward.argtypes = [C.c_void_p] + [C.c_int] * 7 + [C.c_void_p] * 8
        f = _c(faces, np.int32).reshape(-1)
        tc = _c(texcoords, np.float32).reshape(-1)
        self.N, self.C, self.W, self.H = N, C_, W, H
        self.h = L.hcref_uv_create(N, _p(f), f.size // 3, _p(tc), C_, W, H, albedo.encode(), shading.encode(),
                                   normal_mode.encode())

    def forward(self, B, verts, extr, intr, TH, TW):
        import torch
        dev = verts.device
        o = {"bary": torch.full((B, self.C, self.H, self.W, 2), 7.0, device=dev),
             "face": torch.full((B, self.C, self.H, self.W), 7, device=dev, dtype=torch.int32),
             "render": torch.full((B, self.C, self.H, self.W, 3), 7.0, device=dev),
             "vnormal": torch.zeros((B, self.C, self.N, 3), device=dev),
             "normal_map": torch.zeros((B, TH, TW, 3), device=dev)}
        torch.cuda.synchronize()
        st = ref_lib().hcref_uv_forward(self.h, B, self.N, self.C, self.W, self.H, TW, TH, _p(verts), _p(extr),
                                        _p(intr), _p(o["bary"]), _p(o["face"]), _p(o["render"]), _p(o["vnormal"]),
                                        _p(o["normal_map"]))
        if st != 0:
            raise RuntimeError(f"reference uv forward failed: {st}")
        return o


def texel_table(texcoords, TH, TW):
    """FP64 restatement of the reference's texel table (CUDABasedRasterization.cpp:266-330):
    per texel (face, a, b, c) of the last (largest-id) face whose UV triangle
    contains the texel centre; (0, 0, 0, 0) elsewhere."""
    tc = np.asarray(texcoords, np.float64).reshape(-1, 3, 2)
    F = tc.shape[0]
    out = np.zeros((TH, TW, 4))
    for f in range(F):
        p = np.stack([TW * tc[f, :, 0], TH * (1.0 - tc[f, :, 1])], 1)
        x0 = int(max(p[:, 0].min() - 2, 0))
        x1 = int(min(p[:, 0].max() + 2, TW))
        y0 = int(max(p[:, 1].min() - 2, 0))
        y1 = int(min(p[:, 1].max() + 2, TH))
        if x1 <= x0 or y1 <= y0:
            continue
        xx, yy = np.meshgrid(np.arange(x0, x1) + 0.5, np.arange(y0, y1) + 0.5)
        e = lambda a, b, px, py: (b[0] - a[0]) * (py - a[1]) - (b[1] - a[1]) * (px - a[0])  # noqa: E731
        nz = e(p[0], p[1], p[2][0], p[2][1])
        if nz == 0:
            continue
        s0 = e(p[0], p[1], xx, yy) * nz
        a = e(p[1], p[2], xx, yy) * nz
        b = e(p[2], p[0], xx, yy) * nz
        hit = (s0 >= 0) & (a >= 0) & (b >= 0)
        aa, bb = a / (nz * nz), b / (nz * nz)
        sl = out[y0:y1, x0:x1]
        sl[hit] = np.stack([np.full(hit.sum(), f), aa[hit], bb[hit], 1 - aa[hit] - bb[hit]], 1)
    return out


# ---------------------------------------------------------------------------
# host kinematics in float, the reference's procedure (hc_oracle_fk.inc)
# ---------------------------------------------------------------------------
def fk_f32(ch, dofs):
    """Global joint positions / axes [B,J,3] and skinning-joint dual
    quaternions [B,S,8] by the reference's dual-quaternion joint chain in float."""
    i32 = lambda a: _c(a, np.int32)  # noqa: E731
    f32 = lambda a: None if a is None else _c(a, np.float32)  # noqa: E731
    dofs = f32(np.atleast_2d(dofs))
    B, J, S, D = dofs.shape[0], ch.n_joints, ch.n_skin, ch.n_dofs
    arr = [i32(ch.parent), i32(ch.joint_type), f32(ch.offset), f32(ch.axis), f32(ch.joint_scale),
           i32(ch.dof_offsets), i32(ch.dof_joint), f32(ch.dof_weight), i32(ch.skin_joint), f32(ch.skin_scale)]
    pos, ax, dq = np.zeros((B, J, 3), np.float32), np.zeros((B, J, 3), np.float32), np.zeros((B, S, 8), np.float32)
    fn = oracle_lib().hco_fk_f32
    vp_ = C.c_void_p
    p = lambda a: vp_(None) if a is None else vp_(_p(a))  # noqa: E731
    st = fn(B, J, p(arr[0]), p(arr[1]), p(arr[2]), p(arr[3]), p(arr[4]), D, p(arr[5]), p(arr[6]), p(arr[7]), S,
            p(arr[8]), p(arr[9]), p(dofs), p(pos), p(ax), p(dq))
    if st != 0:
        raise RuntimeError("oracle fk failed")
    return pos, ax, dq


def pose2eg_f32(ch, dq, node_vertex, weights):
    """Pose2EmbeddedGraphCpu's node blend + Euler angles in float on the given
    joint dual quaternions [B,S,8]: (skinned_t, skinned_a) [B,M,3]."""
    dq = _c(dq, np.float32)
    nv = _c(node_vertex, np.int32)
    si, w = _c(ch.skin_index, np.int32), _c(weights, np.float32)
    B, S = dq.shape[:2]
    N, K = si.shape
    M = nv.shape[0]
    t, a = np.zeros((B, M, 3), np.float32), np.zeros((B, M, 3), np.float32)
    vp_ = C.c_void_p
    st = oracle_lib().hco_pose2eg_f32(B, S, N, K, vp_(_p(si)), vp_(_p(w)), M, vp_(_p(nv)), vp_(_p(dq)), vp_(_p(t)),
                                      vp_(_p(a)))
    if st != 0:
        raise RuntimeError("oracle pose2eg failed")
    return t, a
