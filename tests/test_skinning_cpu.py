"""Forward-kinematics / skinning oracle self-checks (no GPU).

Eigen and the character loaders are not available, so the reference host
kinematics cannot run here; the FP64 restatement is pinned by identities
(zero pose, rigid motions) and finite differences instead."""
import numpy as np
import pytest

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.skinning import Character
from oracle import skinning_oracle as K


@pytest.fixture(scope="module")
def scene():
    sc = S.skinning_scene(2, 6, batch=2, seed=3)
    ch = Character.from_synthetic(sc["skeleton"], sc["verts"], sc["faces"], sc["skin_index"])
    return sc, ch


def test_zero_pose_is_identity(scene):
    sc, ch = scene
    dq = K.dual_quaternions(ch, np.zeros((1, ch.n_dofs)))
    np.testing.assert_allclose(dq[0, :, :4], np.tile([0, 0, 0, 1.0], (ch.n_skin, 1)), atol=1e-12)
    np.testing.assert_allclose(dq[0, :, 4:], 0, atol=1e-9)
    v, n = K.dq_skin(ch, dq, sc["weights"][:1])
    np.testing.assert_allclose(v[0], ch.base_vertices, atol=1e-9)
    np.testing.assert_allclose(n[0], ch.base_normals, atol=1e-6)


def test_dual_quaternion_reproduces_matrix_transform(scene):
    sc, ch = scene
    Rs, ts = K.skin_transforms(ch, sc["dofs"])
    dq = K.dual_quaternions(ch, sc["dofs"])
    for b in range(2):
        for s in range(ch.n_skin):
            np.testing.assert_allclose(K.quat_rot(dq[b, s, :4]), Rs[b, s], atol=1e-12)
            np.testing.assert_allclose(K.dq_trans(dq[b, s, :4], dq[b, s, 4:]), ts[b, s], atol=1e-9)


def test_single_bone_vertex_moves_rigidly(scene):
    """A vertex weighted 1 to one bone follows that bone's transform exactly (DQ and LBS)."""
    sc, ch = scene
    w = np.zeros_like(sc["weights"][:1])
    w[..., 0] = 1.0
    dq = K.dual_quaternions(ch, sc["dofs"][:1])
    v, _ = K.dq_skin(ch, dq, w)
    Rs, ts = K.skin_transforms(ch, sc["dofs"][:1])
    lv, _ = K.lbs_skin(ch, Rs, ts, w, np.zeros((1, ch.base_vertices.shape[0], 3)))
    bone = ch.skin_index[:, 0]
    expect = np.einsum("vij,vj->vi", Rs[0, bone], ch.base_vertices) + ts[0, bone]
    np.testing.assert_allclose(v[0], expect, atol=1e-6)
    np.testing.assert_allclose(lv[0], expect, atol=1e-6)


def test_reference_dof_gradient_is_exact_for_rigid_vertices(scene):
    """The reference's linearised dof gradient sum w (axis x (v - c)) . g equals the
    true derivative when every vertex follows a single bone."""
    sc, ch = scene
    w = np.zeros_like(sc["weights"][:1])
    w[..., 0] = 1.0
    dofs = sc["dofs"][:1].astype(np.float64)
    rng = np.random.default_rng(0)
    g = rng.normal(size=(1, ch.base_vertices.shape[0], 3))

    def loss(d):
        Rs, ts = K.skin_transforms(ch, d)
        v, _ = K.lbs_skin(ch, Rs, ts, w, np.zeros_like(g))
        return float((v * g).sum())

    Rs, ts = K.skin_transforms(ch, dofs)
    v, _ = K.lbs_skin(ch, Rs, ts, w, np.zeros_like(g))
    _, _, gpos, gaxis = K.fk(ch, dofs)
    ana = K.dof_grad_reference(ch, v, g, w, gpos, gaxis)
    h = 1e-6
    for d in rng.choice(ch.n_dofs, 5, replace=False):
        p, m = dofs.copy(), dofs.copy()
        p[0, d] += h
        m[0, d] -= h
        fd = (loss(p) - loss(m)) / (2 * h)
        assert abs(fd - ana[0, d]) <= 1e-4 * max(1.0, abs(fd)), (d, fd, ana[0, d])
