"""Pinning of the host kinematics and the node skinning: two independent
restatements of the reference, checked against each other.

* oracle/hc_oracle_fk.inc follows the reference's own procedure in float:
  per joint, the parent's transform and the local (offset, axis-angle)
  transform become dual quaternions, are multiplied and normalised, and
  come back to a matrix (Skeletool/Character/joint.cpp:36-116 with
  DualQuaternion.h), then joint x scale x inverse(bind) becomes each skinning
  joint's dual quaternion (DQSkinningGPUOp.cpp:257-300), and the node loop of
  Pose2EmbeddedGraphCPUOp.cpp:196-290 blends them and extracts Z-Y-X Euler
  angles.
* oracle/skinning_oracle.py composes plain rotation matrices in FP64.

The two must agree to float rounding: joint positions, axes, dual
quaternions (up to the sign of q), node translations and angles.
"""
import numpy as np
import pytest

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.chain import character
from oracle import oracle as O
from oracle import skinning_oracle as K


def wrap(a):
    return np.arctan2(np.sin(a), np.cos(a))


@pytest.mark.parametrize("scaled", [False, True])
def test_float_dq_chain_matches_fp64_matrix_chain(scaled):
    sc = S.chain_scene(3, 120, 24, 4, 1, 32, 32, seed=7, pose_amplitude=1.5)
    ch = character(sc)
    if scaled:  # non-unit joint and skinning-joint scales (the loaders' characters have them)
        rng = np.random.default_rng(3)
        ch.joint_scale = rng.uniform(0.8, 1.25, ch.n_joints).astype(np.float32)
        ch.skin_scale = rng.uniform(0.8, 1.25, ch.n_skin).astype(np.float32)
    dofs = sc["dofs"]
    pos, ax, dq = O.fk_f32(ch, dofs)
    _, t64, p64, a64 = K.fk(ch, dofs)
    assert np.abs(pos - p64).max() < 1e-5 * np.abs(p64).max()  # float rounding over the joint chain
    assert np.abs(ax - a64).max() < 1e-5
    dq64 = K.dual_quaternions(ch, dofs)
    sign = np.where((dq[..., :4] * dq64[..., :4]).sum(-1, keepdims=True) < 0, -1.0, 1.0)
    assert np.abs(dq[..., :4] * sign - dq64[..., :4]).max() < 1e-5
    assert np.abs(dq[..., 4:] * sign - dq64[..., 4:]).max() < 1e-5 * np.abs(dq64[..., 4:]).max()


def test_float_node_skinning_matches_fp64():
    sc = S.chain_scene(3, 120, 24, 4, 1, 32, 32, seed=8)
    ch = character(sc)
    nodes = sc["graph"].node_vertex
    _, _, dq = O.fk_f32(ch, sc["dofs"])
    t32, a32 = O.pose2eg_f32(ch, dq, nodes, sc["skin_weights"])
    t64, a64, _ = K.pose2eg(ch, sc["dofs"], nodes, sc["skin_weights"])
    assert np.abs(t32 - t64).max() < 1e-5 * np.abs(t64).max()
    assert np.abs(wrap(a32 - a64)).max() < 1e-4
    assert np.abs(t64).max() > 10.0 and np.abs(a64).max() > 0.1


def test_zero_pose_is_the_bind_pose():
    sc = S.chain_scene(2, 40, 8, 1, 1, 16, 16, seed=2)
    ch = character(sc)
    _, _, dq = O.fk_f32(ch, np.zeros((1, ch.n_dofs), np.float32))
    assert np.abs(np.abs(dq[..., 3]) - 1.0).max() < 1e-6
    assert np.abs(dq[..., :3]).max() < 1e-6 and np.abs(dq[..., 4:]).max() < 1e-3
