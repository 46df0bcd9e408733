"""Host logic of the chain: every C-ABI call that one step issues names an
exported symbol with the declared number of arguments, in the order of the
reference's TF graph (no GPU: the library calls are recorded, not run)."""
import numpy as np
import pytest

from deepcharacters_b200 import _lib
from deepcharacters_b200 import synthetic as S


@pytest.fixture
def recorder(monkeypatch):
    calls = []

    def fake_call(name, *args):
        assert name in _lib._SIGS, name
        assert len(args) == len(_lib._SIGS[name]), (name, len(args), len(_lib._SIGS[name]))
        calls.append((name, args))

    monkeypatch.setattr(_lib, "call", fake_call)
    import deepcharacters_b200.chain as chain
    monkeypatch.setattr(chain, "_stream", lambda: 0)
    return calls


def test_chain_step_calls(recorder):
    from deepcharacters_b200.chain import DeformRenderChain
    sc = S.chain_scene(1, 12, 2, 2, 2, 32, 32, seed=3)
    ch = DeformRenderChain(sc, "cpu", 2, 2, 32, 32)
    recorder.clear()
    ch.step()
    names = [n for n, _ in recorder]
    assert names == ["hc_pose2eg_forward", "hc_eg_forward", "hc_renderer_forward_l1",
                     "hc_camera_projection_forward", "hc_camera_projection_forward", "hc_mesh_boundary_forward_hinted",
                     "hc_silhouette_forward_sumsq_sized", "hc_sum_squares_loss", "hc_silhouette_backward_scaled_sized",
                     "hc_camera_projection_backward", "hc_renderer_backward_l1", "hc_add_inplace", "hc_eg_backward",
                     "hc_pose2eg_backward"]
    args = dict(recorder)
    # the EG consumes the node transforms that the node skinning wrote
    assert args["hc_eg_forward"][5] == args["hc_pose2eg_forward"][7]
    assert args["hc_eg_forward"][6] == args["hc_pose2eg_forward"][8]
    # the raster and the silhouette see the EG vertices; the summed gradient feeds the EG adjoint
    v = args["hc_eg_forward"][8]
    assert args["hc_renderer_forward_l1"][3] == v and args["hc_camera_projection_forward"][4] == v
    assert args["hc_eg_backward"][3] == args["hc_renderer_backward_l1"][18] == args["hc_add_inplace"][2]
    # the fused L1: the adjoint reads the state and the render buffer the forward wrote
    assert args["hc_renderer_backward_l1"][3] == args["hc_renderer_forward_l1"][17]
    assert args["hc_renderer_backward_l1"][4] == args["hc_renderer_forward_l1"][13]
    # the mesh boundary takes the renderer's face buffer as its coverage hint
    assert args["hc_mesh_boundary_forward_hinted"][10] == args["hc_renderer_forward_l1"][12]
    assert args["hc_add_inplace"][3] == args["hc_camera_projection_backward"][9]
    # joint angles: the EG's skinned-transform gradients feed the node-skinning adjoint
    assert args["hc_pose2eg_backward"][7] == args["hc_eg_backward"][9]
    assert args["hc_pose2eg_backward"][8] == args["hc_eg_backward"][10]
    # the per-pixel residual's squared loss is fused into the silhouette forward, and
    # its adjoint reads the residual itself with the factor 2 w1
    fw, bw = args["hc_silhouette_forward_sumsq_sized"], args["hc_silhouette_backward_scaled_sized"]
    assert bw[7] == fw[13] and abs(bw[8] - 2 * ch.w_sil1) < 1e-12 and fw[16] == ch.w_sil1
    assert args["hc_sum_squares_loss"][1] == 2 * 2 * sc["N"]
    assert np.isfinite(sc["dofs"]).all()


def test_chain_step_calls_mixed_sizes_vertex_dq(recorder):
    """Cameras of different sizes and per-vertex DQ skinning: the sized
    boundary / silhouette entry points with the per-camera size arrays, flat
    per-pixel buffers of a frame, and the DQ adjoint fed by the summed vertex
    gradient."""
    from deepcharacters_b200.chain import DeformRenderChain
    ws, hs = [32, 48, 64], [32, 64, 48]
    sc = S.chain_scene(1, 12, 4, 2, 3, ws, hs, seed=3)
    assert sc["dt"].shape == (2, sum(w * h for w, h in zip(ws, hs)))
    ch = DeformRenderChain(sc, "cpu", 2, 3, ws, hs, deformation="dq")
    assert ch.multires and ch.buf["face"].shape == (2, ch.P_frame) and ch.buf["res1"].shape == (2, ch.P_frame, 2)
    recorder.clear()
    ch.step()
    names = [n for n, _ in recorder]
    assert names == ["hc_dq_skinning_forward", "hc_renderer_forward_l1", "hc_camera_projection_forward",
                     "hc_camera_projection_forward", "hc_mesh_boundary_forward_sized",
                     "hc_silhouette_forward_sumsq_sized", "hc_sum_squares_loss", "hc_silhouette_backward_scaled_sized",
                     "hc_camera_projection_backward", "hc_renderer_backward_l1", "hc_add_inplace",
                     "hc_dq_skinning_backward"]
    args = dict(recorder)
    import ctypes
    w = args["hc_mesh_boundary_forward_sized"][4]
    assert list((ctypes.c_int32 * 3).from_address(w)) == ws
    assert list((ctypes.c_int32 * 3).from_address(args["hc_silhouette_forward_sumsq_sized"][5])) == ws
    assert list((ctypes.c_int32 * 3).from_address(args["hc_silhouette_backward_scaled_sized"][5])) == hs
    v = args["hc_dq_skinning_forward"][5]
    assert args["hc_renderer_forward_l1"][3] == v and args["hc_dq_skinning_backward"][4] == v
    assert args["hc_dq_skinning_backward"][3] == args["hc_add_inplace"][2]
