"""Character / skeleton / skin / mesh / graph file loaders (host only).

Files are written here in the reference's formats (Skeletool/Character/
skeleton.cpp:254-530, skinnedcharacter.cpp:149-206, 425-559, Mesh/trimesh.cpp:
337-480) from a synthetic character, read back, and compared with the arrays
they were written from; the embedded graph is compared with the loop-by-loop
restatement in ``oracle/loader_oracle.py``."""
import os

import numpy as np
import pytest

from deepcharacters_b200 import loaders as L
from deepcharacters_b200 import synthetic as S
from deepcharacters_b200.skinning import Character
from oracle import loader_oracle as LO

AX = "xyz"


def _f(x):
    return repr(float(x))


def _names(sk):
    return [f"j{j // 3:02d}_{AX[j % 3]}" for j in range(sk.n_joints)]


def write_character(d, sc, eol="\r\n", scales=None, markers=(), limits=None, segmentation=None, graph=None):
    """Writes skeleton, skin, mesh (+ segmentation, graph mesh) and the .character file into ``d``."""
    sk = sc["skeleton"]
    names = _names(sk)
    J = sk.n_joints
    scales = np.ones(J, np.float32) if scales is None else scales
    L_ = ["Skeletool Skeleton Definition V1.0", f"joints: {J}"]
    for j in range(J):
        p = names[sk.parent[j]] if sk.parent[j] >= 0 else "none"
        o, a = sk.offset[j], sk.axis[j]
        L_.append(f"{names[j]} revolute {p} {_f(o[0])} {_f(o[1])} {_f(o[2])} {_f(a[0])} {_f(a[1])} {_f(a[2])} {_f(scales[j])}")
    L_.append(f"markers: {len(markers)}")
    for i, (jn, off) in enumerate(markers):
        L_.append(f"m{i} {jn} point {_f(off[0])} {_f(off[1])} {_f(off[2])}")
    L_.append("scaling joints: 1")
    L_.append("arm 2")
    L_.append(names[0])
    L_.append(names[3])
    L_.append(f"dofs: {J}")
    for j in range(J):
        L_.append(f"d{j} 1")
        L_.append("nolimits" if limits is None or limits[j] is None else f"limits {limits[j][0]} {limits[j][1]}")
        L_.append(f"{names[j]} 1")
    _write(os.path.join(d, "actor.skeleton"), L_, eol)
    n_skel = J // 3
    w = sc["weights"][0]
    idx = sc["skin_index"]
    K_ = ["Skeletool character skinning file V1.0", "bones:", " ".join(f"j{s:02d}" for s in range(n_skel)),
          "vertex weights:"]
    for v in range(idx.shape[0]):
        K_.append(f"{v} " + " ".join(f"{int(idx[v, k])} {_f(w[v, k])}" for k in range(idx.shape[1])))
    _write(os.path.join(d, "actor.skin"), K_, eol)
    _write_obj(os.path.join(d, "actor.obj"), sc["verts"], sc["faces"], eol)
    if segmentation is not None:
        _write(os.path.join(d, "segmentation.txt"), [str(int(x)) for x in segmentation], "\n")
    if graph is not None:
        _write_obj(os.path.join(d, "graph.obj"), graph[0], graph[1], eol)
    _write(os.path.join(d, "actor.character"),
           ["skeletool character file v1.0", "skeleton", "actor.skeleton", "mesh", "actor.obj", "skin", "actor.skin"],
           eol)
    return os.path.join(d, "actor.character")


def _write(path, lines, eol):
    with open(path, "wb") as fh:
        fh.write((eol.join(lines) + eol).encode())


def _write_obj(path, verts, faces, eol):
    lines = ["# mesh"] + [f"v {_f(p[0])} {_f(p[1])} {_f(p[2])}" for p in np.asarray(verts, np.float32)]
    lines += [f"f {a + 1} {b + 1} {c + 1}" for a, b, c in faces]
    _write(path, lines, eol)


@pytest.fixture(scope="module")
def scene():
    return S.skinning_scene(2, 8, batch=1, seed=23)


def test_character_round_trip(scene, tmp_path):
    sc = scene
    cf = L.load_character(write_character(str(tmp_path), sc))
    ch = cf.character()
    ref = Character.from_synthetic(sc["skeleton"], sc["verts"], sc["faces"], sc["skin_index"])
    for k in ("parent", "joint_type", "offset", "axis", "dof_offsets", "dof_joint", "dof_weight", "skin_joint",
              "base_vertices", "skin_index"):
        np.testing.assert_array_equal(getattr(ch, k), getattr(ref, k), err_msg=k)
    np.testing.assert_allclose(ch.base_normals, ref.base_normals, atol=2e-6)
    np.testing.assert_array_equal(cf.skin_weight, sc["weights"][0])
    np.testing.assert_array_equal(cf.mesh.faces, sc["faces"])
    assert cf.skeleton.joint_names[:3] == ["j00_x", "j00_y", "j00_z"]
    np.testing.assert_array_equal(ch.joint_scale, np.ones(ch.n_joints, np.float32))


def test_lf_and_crlf_read_the_same(scene, tmp_path):
    a, b = tmp_path / "crlf", tmp_path / "lf"
    a.mkdir()
    b.mkdir()
    ca = L.load_character(write_character(str(a), scene, eol="\r\n")).character()
    cb = L.load_character(write_character(str(b), scene, eol="\n")).character()
    for k in ("parent", "offset", "axis", "skin_index", "base_vertices"):
        np.testing.assert_array_equal(getattr(ca, k), getattr(cb, k))


def test_unterminated_last_line_is_not_read(tmp_path):
    p = tmp_path / "x.obj"
    p.write_bytes(b"v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1 2 3\nf 1 2 4")
    m = L.load_obj(str(p))
    assert m.faces.shape == (1, 3)


def test_obj_fan_triangulation_texture_and_normals(tmp_path):
    p = tmp_path / "quad.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0 0.5 0.25 1\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\n"
                 "f 1/1 2/2 3/3 4/4\n")
    m = L.load_obj(str(p))
    np.testing.assert_array_equal(m.faces, [[0, 1, 2], [0, 2, 3]])
    np.testing.assert_array_equal(m.face_tindex, [[0, 1, 2], [0, 2, 3]])
    np.testing.assert_array_equal(m.normals, np.tile([0, 0, 1], (4, 1)).astype(np.float32))
    np.testing.assert_array_equal(m.colors[3], [0.5, 0.25, 1.0])
    np.testing.assert_array_equal(m.colors[0], [1, 1, 1])
    np.testing.assert_array_equal(m.face_uvs()[:6], [0, 0, 1, 0, 1, 1])


def test_name_lookups_follow_the_reference_prefix_rules(scene, tmp_path):
    cf = L.load_character(write_character(str(tmp_path), scene))
    sk = cf.skeleton
    assert sk.joint_by_name("j01") == 3        # first joint starting with the name (dofs, markers)
    assert sk.last_joint_by_name("j01") == 5   # last one (skin bones)
    np.testing.assert_array_equal(cf.skin_joint, 3 * np.arange(8) + 2)


def test_skin_scale_and_bind_pose(scene, tmp_path):
    sk = scene["skeleton"]
    J = sk.n_joints
    scales = (1.0 + 0.05 * np.arange(J)).astype(np.float32)
    lim = [None] * J
    lim[4] = (0.1, 0.5)
    cf = L.load_character(write_character(str(tmp_path), scene, scales=scales, limits=lim,
                                          markers=[("j02_z", (1.0, 2.0, 3.0))]))
    ch = cf.character()
    np.testing.assert_array_equal(ch.joint_scale, scales)
    exp = np.empty(ch.n_skin, np.float32)
    for s, j in enumerate(ch.skin_joint):
        kids = [c for c in range(J) if sk.parent[c] == j]
        if kids:
            exp[s] = scales[kids[0]]
        else:  # base: walk up through zero offsets (the x and y joints of the same skeletal joint)
            b = j
            while sk.parent[b] >= 0 and not np.any(sk.offset[b]):
                b = sk.parent[b]
            exp[s] = scales[b]
    np.testing.assert_array_equal(ch.skin_scale, exp)
    bd = cf.skeleton.bind_dofs()
    assert bd[4] == np.float32(0.1) and bd[0] == 0.0
    # marker at the bind dofs with the joint scales
    R, t = L.joint_transforms(cf.skeleton, bd)
    np.testing.assert_allclose(L.marker_positions(cf.skeleton)[0], R[8] @ [1.0, 2.0, 3.0] + t[8], rtol=1e-6)


def test_graph_matches_loop_restatement(scene, tmp_path):
    sc = scene
    gv, gf = S.icosphere(0)
    gv = (gv * 990.0).astype(np.float32)  # a coarse shell just inside the mesh
    rng = np.random.default_rng(5)
    seg = rng.choice([0, 5, 9, 11, 14, 2], size=sc["verts"].shape[0])
    cpath = write_character(str(tmp_path), sc, segmentation=seg, graph=(gv, gf),
                            markers=[("j00_z", (0.0, 0.0, 0.0)), ("j03_z", (5.0, 0.0, 0.0))])
    cf = L.load_character(cpath)
    for refinement in (False, True):
        g = L.load_graph(cf, str(tmp_path / "graph.obj"), refinement=refinement)
        seg_w = L.segmentation_weights(cf.mesh_path, cf.mesh.vertices.shape[0])
        o = LO.build_graph(cf.mesh.vertices, cf.mesh.faces, gv, gf, seg_w, L.marker_positions(cf.skeleton),
                           refinement=refinement)
        e = g.eg
        np.testing.assert_array_equal(e.node_vertex, o["node_vertex"])
        np.testing.assert_array_equal(g.radius, o["radius"])
        for v, c in enumerate(o["conn"]):
            a, n = e.v2n_offsets[v], e.v2n_sizes[v]
            np.testing.assert_array_equal(e.v2n_indices[a:a + n], [i for i, _ in c])
            np.testing.assert_array_equal(e.v2n_weights[a:a + n], np.array([w for _, w in c], np.float32))
        for k, lst in enumerate(o["n2v"]):
            a, n = e.n2v_offsets[k], e.n2v_sizes[k]
            np.testing.assert_array_equal(e.n2v_indices[a:a + n], [v for v, _ in lst])
            np.testing.assert_array_equal(e.n2v_weights[a:a + n], np.array([w for _, w in lst], np.float32))
        for k, lst in enumerate(o["n2n"]):
            a, n = g.n2n_offsets[k], g.n2n_sizes[k]
            np.testing.assert_array_equal(g.n2n_indices[a:a + n], lst)
        np.testing.assert_array_equal(g.rigidity, np.array(o["rigidity"], np.float32))
        np.testing.assert_array_equal(e.marker_node, o["marker_node"])
    assert g.max_connections == 5
    np.testing.assert_allclose(np.add.reduceat(e.v2n_weights, e.v2n_offsets), 1.0, atol=1e-6)


def test_loader_errors(scene, tmp_path):
    cpath = write_character(str(tmp_path), scene, segmentation=[3] * 10 + [99] * 200)
    (tmp_path / "bad.skeleton").write_text("Skeleton v0.3\n")
    with pytest.raises(NotImplementedError):
        L.load_skeleton(str(tmp_path / "bad.skeleton"))
    (tmp_path / "bad2.skeleton").write_text("hello\n")
    with pytest.raises(ValueError):
        L.load_skeleton(str(tmp_path / "bad2.skeleton"))
    with pytest.raises(ValueError, match="segmentation category 99"):
        L.segmentation_weights(os.path.join(str(tmp_path), "actor.obj"), 20)
    txt = open(cpath, "rb").read() + b"pose\r\nactor.pose\r\n"
    (tmp_path / "posed.character").write_bytes(txt)
    with pytest.raises(NotImplementedError):
        L.load_character(str(tmp_path / "posed.character"))
    with pytest.raises(NotImplementedError):
        L.load_skin(str(tmp_path / "actor.pskin"), None)
