"""ctypes binding of ``libhc.so`` (the C ABI in ``include/hc.h``).

The library is built in-tree by ``deepcharacters_b200.build``.  There is no
fallback: if the library is missing or fails to load, every op raises.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libhc.so")

_lib = None

c_int_p = C.POINTER(C.c_int32)
c_i64_p = C.POINTER(C.c_int64)
vp = C.c_void_p

# name -> argument types (all functions return hc_status / int32 unless listed)
_SIGS: dict[str, list] = {
    "hc_renderer_create": [C.POINTER(vp), vp, C.c_int32, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                           C.c_int32, C.c_char_p, C.c_char_p, C.c_int32, C.c_int32, C.c_char_p],
    "hc_renderer_destroy": [vp],
    "hc_renderer_reserve": [vp, C.c_int32],
    "hc_renderer_set_tuning": [vp, C.c_int32, C.c_int32],
    "hc_renderer_forward": [vp, vp, C.c_int32, vp, vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp, vp, vp],
    "hc_renderer_forward_l1": [vp, vp, C.c_int32, vp, vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp, vp, vp,
                               vp, vp, vp],
    "hc_renderer_backward_l1": [vp, vp, C.c_int32, vp, vp, vp, vp, vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, vp,
                                vp, vp, vp, vp, vp, vp],
    "hc_renderer_forward_ex": [vp, vp, C.c_int32, vp, vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp, vp,
                               vp, vp, vp],
    "hc_renderer_stats": [vp, vp, c_i64_p, c_i64_p],
    "hc_renderer_set_gradient_parity": [vp, C.c_int32],
    "hc_renderer_set_adjoint_schedule": [vp, C.c_int32],
    "hc_eg_create": [C.POINTER(vp), C.c_int32, vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                     C.c_int32, vp, vp],
    "hc_eg_destroy": [vp],
    "hc_eg_reserve": [vp, C.c_int32],
    "hc_eg_set_full_skinned_gradient": [vp, C.c_int32],
    "hc_eg_forward": [vp, vp, C.c_int32] + [vp] * 11,
    "hc_eg_backward": [vp, vp, C.c_int32] + [vp] * 11,
    "hc_arap_create": [C.POINTER(vp), C.c_int32, vp, C.c_int32, vp, vp, vp, vp, vp, C.c_int32],
    "hc_arap_destroy": [vp],
    "hc_arap_forward": [vp, vp, C.c_int32, vp, vp, vp, vp, vp],
    "hc_arap_backward": [vp, vp, C.c_int32, vp, vp, vp, vp],
    "hc_skin_create": [C.POINTER(vp), C.c_int32, vp, vp, vp, vp, vp, C.c_int32, vp, vp, vp, C.c_int32, vp, vp,
                       C.c_int32, vp, vp, C.c_int32, vp],
    "hc_skin_destroy": [vp],
    "hc_skin_reserve": [vp, C.c_int32],
    "hc_skin_set_parity": [vp, C.c_int32],
    "hc_dq_skinning_forward": [vp, vp, C.c_int32] + [vp] * 8,
    "hc_dq_skinning_backward": [vp, vp, C.c_int32] + [vp] * 8,
    "hc_lb_skinning_forward": [vp, vp, C.c_int32] + [vp] * 9,
    "hc_lb_skinning_backward": [vp, vp, C.c_int32] + [vp] * 10,
    "hc_camera_projection_forward": [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, C.c_int32, vp],
    "hc_camera_projection_backward": [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, C.c_int32, vp],
    "hc_projected_mesh_boundary": [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp],
    "hc_silhouette_create": [C.POINTER(vp)],
    "hc_silhouette_destroy": [vp],
    "hc_silhouette_reserve": [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32],
    "hc_silhouette_forward": [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32] + [vp] * 9,
    "hc_silhouette_forward_static": [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32] + [vp] * 9,
    "hc_silhouette_backward": [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32] + [vp] * 6,
    "hc_pose2eg_forward": [vp, vp, C.c_int32, vp, C.c_int32, vp, vp, vp, vp, vp],
    "hc_pose2eg_backward": [vp, vp, C.c_int32, vp, C.c_int32, vp, vp, vp, vp, vp],
    "hc_mesh_boundary_create": [vp, vp, C.c_int32, C.c_int32],
    "hc_mesh_boundary_destroy": [vp],
    "hc_mesh_boundary_reserve": [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32],
    "hc_mesh_boundary_forward": [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, vp],
    "hc_mesh_boundary_forward_hinted": [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, vp,
                                        vp],
    "hc_mesh_boundary_reserve_sized": [vp, C.c_int32, C.c_int32, vp, vp],
    "hc_mesh_boundary_forward_sized": [vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp, vp, vp],
    "hc_silhouette_reserve_sized": [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp],
    "hc_silhouette_forward_sized": [vp, vp, C.c_int32, C.c_int32, C.c_int32, vp, vp] + [vp] * 9,
    "hc_silhouette_backward_sized": [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp] + [vp] * 6,
    "hc_silhouette_forward_sumsq_sized": [vp, vp, C.c_int32, C.c_int32, C.c_int32, vp, vp] + [vp] * 9
    + [C.c_float, vp, vp],
    "hc_silhouette_backward_scaled_sized": [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp, C.c_float,
                                            vp, vp, vp, vp],
    "hc_sum_squares_loss": [vp, C.c_int64, vp, C.c_float, vp, vp, vp],
    "hc_add_inplace": [vp, C.c_int64, vp, vp],
    "hc_image_u8_to_f32": [vp, C.c_int64, vp, vp],
    "hc_gaussian_smooth": [vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_float, vp, vp],
    "hc_renderer_set_kernel_timing": [vp, C.c_int32],
    "hc_renderer_create_multires": [vp, vp, C.c_int32, vp, C.c_int32, C.c_int32, C.c_int32, vp, vp, C.c_char_p,
                                    C.c_char_p, C.c_int32, C.c_int32, C.c_char_p],
    "hc_renderer_frame_pixels": [vp, vp],
    "hc_renderer_kernel_times": [vp, vp, C.c_int32],
    "hc_image_l1_loss": [vp, C.c_int64, vp, vp, vp, vp, vp, vp, vp],
    "hc_renderer_backward": [vp, vp, C.c_int32, vp, vp, vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, vp, vp, vp,
                             vp, vp, vp, vp],
}

_RESTYPES = {"hc_last_error": C.c_char_p, "hc_version": C.c_char_p, "hc_kernel_launches": C.c_int64}


class HcError(RuntimeError):
    """A C-ABI call returned a non-zero hc_status."""

    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} failed (status {status}): {msg}")
        self.status = status


def lib() -> C.CDLL:
    """Load libhc.so once; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m deepcharacters_b200.build`")
    L = C.CDLL(LIB_PATH)
    for name, rt in _RESTYPES.items():
        getattr(L, name).restype = rt
        getattr(L, name).argtypes = []
    for name, args in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int32
    _lib = L
    return L


def declared_symbols() -> list[str]:
    return list(_SIGS) + list(_RESTYPES)


def call(name: str, *args) -> None:
    st = getattr(lib(), name)(*args)
    if st != 0:
        msg = lib().hc_last_error().decode(errors="replace")
        raise HcError(name, st, msg)


def ptr(t) -> int | None:
    """Device (or host) address of a tensor / array, None for None."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data
