"""Device forward kinematics + DQ / LBS skinning against the FP64 oracle and
the reference skinning kernels (fed with the same dual quaternions /
transforms, since the reference computes those on the host with Eigen)."""
import numpy as np
import pytest
import torch

from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.skinning import Character, SkinningEngine, dq_skinning_gpu, lb_skinning_gpu
from oracle import oracle as O
from oracle import skinning_oracle as K

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference kernels (oracle/_ref) not built")


def _t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(DEV)


def nrel(a, b):
    a = torch.as_tensor(a).double().cpu()
    b = torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / max(b.norm().item(), 1e-30))


@pytest.fixture(scope="module")
def scene():
    sc = S.skinning_scene(4, 24, batch=3, seed=17)
    ch = Character.from_synthetic(sc["skeleton"], sc["verts"], sc["faces"], sc["skin_index"])
    return sc, ch


def test_fk_and_dq_match_fp64_oracle(scene):
    sc, ch = scene
    eng = SkinningEngine(ch)
    v, n, gp, ga, dq, w = eng.dq_forward(_t(sc["dofs"]), _t(sc["weights"]))
    _, _, gpos, gaxis = K.fk(ch, sc["dofs"])
    assert nrel(gp, gpos) < 1e-5 and nrel(ga, gaxis) < 1e-5
    dq_o = K.dual_quaternions(ch, sc["dofs"])
    assert np.abs(dq.cpu().numpy() - dq_o).max() < 1e-4
    vo, no = K.dq_skin(ch, dq_o, sc["weights"])
    assert nrel(v, vo) < 1e-5 and nrel(n, no) < 1e-5
    assert torch.equal(w, _t(sc["weights"]))


@needs_ref
def test_dq_skinning_matches_reference_kernels(scene):
    sc, ch = scene
    eng = SkinningEngine(ch)
    w = _t(sc["weights"])
    v, n, gp, ga, dq, _ = eng.dq_forward(_t(sc["dofs"]), w)
    ref = O.RefSkin(ch)
    rv, rn, rdq, rw = ref.dq_forward(dq, w)
    torch.cuda.synchronize()
    assert torch.equal(v, rv) and torch.equal(n, rn) and torch.equal(dq, rdq)
    g = torch.randn(v.shape, device=DEV, generator=torch.Generator(DEV).manual_seed(1))
    gd, gw = eng.dq_backward(g, v, gp, ga, dq, w)
    rgd, rgw = ref.dq_backward(g, v, gp, ga, dq, w, sc["weights"][0])
    assert nrel(gd, rgd) < 1e-5, nrel(gd, rgd)
    assert nrel(gw, rgw) < 1e-5, nrel(gw, rgw)


@needs_ref
def test_lbs_skinning_matches_reference_kernels(scene):
    sc, ch = scene
    eng = SkinningEngine(ch)
    w, disp = _t(sc["weights"]), _t(sc["disp"])
    v, n, gp, ga, xf, _ = eng.lbs_forward(_t(sc["dofs"]), w, disp)
    ref = O.RefSkin(ch)
    rv, rn, rxf, _ = ref.lbs_forward(xf.cpu().numpy(), w, disp)
    torch.cuda.synchronize()
    assert torch.equal(xf, rxf)
    assert nrel(v, rv) < 1e-6 and nrel(n, rn) < 1e-6
    g = torch.randn(v.shape, device=DEV, generator=torch.Generator(DEV).manual_seed(2))
    gd, gw, gdisp = eng.lbs_backward(g, v, gp, ga, xf, w)
    rgd, rgw, rgdisp = ref.lbs_backward(g, v, gp, ga, xf, w, sc["weights"][0])
    assert nrel(gd, rgd) < 1e-5
    assert nrel(gw, rgw) < 1e-5
    assert nrel(gdisp, rgdisp) < 1e-5


def test_exact_weight_and_displacement_gradients_match_finite_differences(scene):
    """With parity off, the weight / displacement gradients are the true derivatives."""
    sc, ch = scene
    eng = SkinningEngine(ch, parity=False)
    B = 1
    dofs, w, disp = sc["dofs"][:B], sc["weights"][:B].astype(np.float64), sc["disp"][:B].astype(np.float64)
    g = np.random.default_rng(3).normal(size=(B, ch.base_vertices.shape[0], 3))
    v, n, gp, ga, dq, _ = eng.dq_forward(_t(dofs), _t(w))
    _, gw = eng.dq_backward(_t(g), v, gp, ga, dq, _t(w))
    vl, nl, gpl, gal, xf, _ = eng.lbs_forward(_t(dofs), _t(w), _t(disp))
    _, lgw, lgd = eng.lbs_backward(_t(g), vl, gpl, gal, xf, _t(w), _t(disp))
    dq_o = K.dual_quaternions(ch, dofs)
    Rs, ts = K.skin_transforms(ch, dofs)
    rng = np.random.default_rng(4)
    h = 1e-6
    for _ in range(6):
        vi, k = int(rng.integers(0, ch.base_vertices.shape[0])), int(rng.integers(0, 4))
        wp, wm = w.copy(), w.copy()
        wp[0, vi, k] += h
        wm[0, vi, k] -= h
        fd = ((K.dq_skin(ch, dq_o, wp)[0] - K.dq_skin(ch, dq_o, wm)[0])[0, vi] @ g[0, vi]) / (2 * h)
        assert abs(fd - float(gw[0, vi, k])) <= 1e-3 * max(1.0, abs(fd)), ("dq", fd, float(gw[0, vi, k]))
        fl = ((K.lbs_skin(ch, Rs, ts, wp, disp)[0] - K.lbs_skin(ch, Rs, ts, wm, disp)[0])[0, vi] @ g[0, vi]) / (2 * h)
        assert abs(fl - float(lgw[0, vi, k])) <= 1e-3 * max(1.0, abs(fl)), ("lbs", fl, float(lgw[0, vi, k]))
    Rb = np.einsum("vk,vkij->vij", w[0], Rs[0, ch.skin_index])
    np.testing.assert_allclose(lgd[0].cpu().numpy(), np.einsum("vji,vj->vi", Rb, g[0]), rtol=1e-4, atol=1e-4)


def test_autograd_wrappers(scene):
    sc, ch = scene
    eng = SkinningEngine(ch)
    dofs = _t(sc["dofs"]).requires_grad_(True)
    w = _t(sc["weights"]).requires_grad_(True)
    disp = _t(sc["disp"]).requires_grad_(True)
    out = dq_skinning_gpu(eng, dofs, w)
    out[0].sum().backward()
    assert dofs.grad is not None and w.grad is not None
    out = lb_skinning_gpu(eng, dofs, w, disp)
    out[0].square().sum().backward()
    assert disp.grad is not None and float(disp.grad.abs().sum()) > 0


def _euler_to_rot(a):
    """R = Rz(z) Ry(y) Rx(x) for Euler angles [...,3] (the convention the EG op reads)."""
    x, y, z = a[..., 0], a[..., 1], a[..., 2]
    cx, sx, cy, sy, cz, sz = np.cos(x), np.sin(x), np.cos(y), np.sin(y), np.cos(z), np.sin(z)
    R = np.empty(a.shape[:-1] + (3, 3))
    R[..., 0, 0] = cz * cy
    R[..., 0, 1] = cz * sy * sx - sz * cx
    R[..., 0, 2] = cz * sy * cx + sz * sx
    R[..., 1, 0] = sz * cy
    R[..., 1, 1] = sz * sy * sx + cz * cx
    R[..., 1, 2] = sz * sy * cx - cz * sx
    R[..., 2, 0] = -sy
    R[..., 2, 1] = cy * sx
    R[..., 2, 2] = cy * cx
    return R


def test_pose2eg_matches_fp64_oracle_and_dq_skinning(scene):
    sc, ch = scene
    eng = SkinningEngine(ch)
    rng = np.random.default_rng(7)
    nodes = rng.choice(ch.base_vertices.shape[0], size=97, replace=False).astype(np.int32)
    w0 = sc["weights"][0]
    t, a, dq = eng.pose2eg(_t(sc["dofs"]), torch.from_numpy(nodes).to(DEV), _t(w0))
    to, ao, dqo = K.pose2eg(ch, sc["dofs"], nodes, w0)
    assert nrel(t, to) < 1e-5
    # angles compared on the circle; the rotation they encode compared directly
    d = a.cpu().double().numpy() - ao
    assert np.abs(np.arctan2(np.sin(d), np.cos(d))).max() < 1e-4
    assert np.abs(_euler_to_rot(a.cpu().double().numpy()) - _euler_to_rot(ao)).max() < 1e-5
    # same dual quaternions as the skinning op, and a node moves like its skinned base vertex
    v, _, _, _, dq_s, _ = eng.dq_forward(_t(sc["dofs"]), _t(sc["weights"]))
    assert torch.equal(dq, dq_s)
    R = _euler_to_rot(a.cpu().double().numpy())
    p = np.einsum("bmij,mj->bmi", R, ch.base_vertices[nodes].astype(np.float64)) + t.cpu().double().numpy()
    assert nrel(p, v[:, torch.from_numpy(nodes).long()]) < 1e-5


def test_pose2eg_rejects_bad_nodes(scene):
    sc, ch = scene
    eng = SkinningEngine(ch)
    with pytest.raises(ValueError):
        eng.pose2eg(_t(sc["dofs"]), torch.tensor([0, ch.base_vertices.shape[0]], device=DEV), _t(sc["weights"][0]))


def test_pose2eg_backward_matches_fp64_finite_differences(scene):
    sc, ch = scene
    eng = SkinningEngine(ch)
    rng = np.random.default_rng(11)
    nodes = rng.choice(ch.base_vertices.shape[0], size=61, replace=False).astype(np.int32)
    w0 = sc["weights"][0]
    dofs = sc["dofs"].astype(np.float64)
    B, D = dofs.shape
    gt = rng.normal(size=(B, len(nodes), 3))
    ga = rng.normal(size=(B, len(nodes), 3))
    ours = eng.pose2eg_backward(_t(dofs), torch.from_numpy(nodes).to(DEV), _t(w0), _t(gt), _t(ga)).cpu().double()

    def loss(d):  # per-frame loss of the FP64 restatement
        t, a, _ = K.pose2eg(ch, d, nodes, w0)
        return (gt * t).sum(axis=(1, 2)) + (ga * a).sum(axis=(1, 2))

    h = 1e-6
    fd = np.zeros((B, D))
    for d in range(D):  # frames are independent: perturb one dof of every frame at once
        p, m = dofs.copy(), dofs.copy()
        p[:, d] += h
        m[:, d] -= h
        fd[:, d] = (loss(p) - loss(m)) / (2 * h)
    assert np.abs(fd).max() > 1.0
    assert nrel(ours, fd) < 1e-4, nrel(ours, fd)


def test_device_kinematics_match_the_float_reference_procedure(scene):
    """The device kinematics and node skinning against the float restatement
    of the reference's own procedure (dual-quaternion joint chain and
    Pose2EmbeddedGraphCpu's node loop, oracle/hc_oracle_fk.inc): both in
    float but in different orders of operations (matrix chain on the device,
    dual-quaternion chain there), so they agree to float rounding (~1e-6)."""
    sc, ch = scene
    eng = SkinningEngine(ch)
    _, _, gp, ga, dq, _ = eng.dq_forward(_t(sc["dofs"]), _t(sc["weights"]))
    pos, ax, dq32 = O.fk_f32(ch, sc["dofs"])
    assert nrel(gp, pos) < 1e-5 and nrel(ga, ax) < 1e-5
    d = dq.cpu().numpy()
    sign = np.where((d[..., :4] * dq32[..., :4]).sum(-1, keepdims=True) < 0, -1.0, 1.0)
    assert nrel(d * sign, dq32) < 1e-5
    rng = np.random.default_rng(5)
    nodes = rng.choice(ch.base_vertices.shape[0], size=50, replace=False).astype(np.int32)
    w0 = sc["weights"][0]
    t, a, _ = eng.pose2eg(_t(sc["dofs"]), torch.from_numpy(nodes).to(DEV), _t(w0))
    t32, a32 = O.pose2eg_f32(ch, dq32, nodes, w0)
    assert nrel(t, t32) < 1e-5
    da = a.cpu().numpy().astype(np.float64) - a32
    assert np.abs(np.arctan2(np.sin(da), np.cos(da))).max() < 1e-4
