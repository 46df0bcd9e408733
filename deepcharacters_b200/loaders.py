"""Character, skin, mesh and embedded-graph file loaders.

The reference ops build their characters from files when they are
constructed: ``DqSkinningGpu`` / ``LbSkinningGpu`` read a ``.character`` file
(CustomGPUOperators/DQSkinningOperator/DQSkinningGPUOp.cpp:22-44), and
``EmbeddedGraphGpu`` reads the character plus a graph mesh
(EmbeddedGraphOperator/EmbeddedGraphGPUOp.cpp:22-60).  This module parses the
same files on the host and returns the arrays the device handles take
(``skinning.Character``, ``embedded_graph.EGData`` and the ARAP node graph), so
real capture data drops in where the synthetic scenes are used.

Formats and rules, all from Skeletool (CustomTensorFlowCPPOperators/src/):
  - lines and tokens: StringProcessing/StringProcessing.cpp:5-60 (split on
    single spaces, empty tokens dropped; a last line without a newline is not
    read).  The reference removes the last character of every line on Linux,
    which is the carriage return of the CRLF files it was written for; here a
    trailing carriage return is removed and LF files read the same.
  - ``.character`` v1.0: Character/skinnedcharacter.cpp:425-559 (skeleton,
    mesh and skin paths relative to the character file).
  - skeleton ``Skeletool Skeleton Definition V1.0``: Character/skeleton.cpp:
    254-530 (joints, markers, scaling groups, dofs with limits); joint lookup by
    name prefix (skeleton.cpp:3655-3677).
  - ``.skin``: skinnedcharacter.cpp:149-206 (bone names resolved to the last
    joint whose name starts with them).
  - ``.obj``: Mesh/trimesh.cpp:337-480 (fan triangulation of polygons, optional
    per-vertex colours, texture indices) and area-weighted vertex normals
    (trimesh.cpp:838-857).
  - per-vertex segmentation weights from ``segmentation.txt`` beside the mesh
    (trimesh.cpp:1305-1380).
  - embedded graph: Mesh/EmbeddedGraph.cpp:5-490 (nodes = the closest unused
    mesh vertex of each graph-mesh vertex in the same connected parts; node
    radius = half the largest hop distance to a graph neighbour, at least 3;
    vertex weights exp(-d^2/2) over the hop distance / radius, normalised;
    rigidity = mean segmentation weight of each node's vertices; markers
    attached to the nearest node).

Only the formats the capture data uses are read: character files v1.0,
skeleton files V1.0, ``.skin`` skinning and ``.obj`` meshes.  Other versions,
Pinocchio / Maya / BVH inputs and initial-pose files raise
``NotImplementedError``; malformed files raise ``ValueError`` where the
reference prints a message and carries on.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

from .embedded_graph import EGData
from .skinning import PRISMATIC, REVOLUTE, Character

_UNREACHED = 1000000  # the reference's "no path" hop distance (trimesh.cpp:868-890)


def _read_lines(path: str) -> list[str]:
    """Lines as the reference's getline loop sees them (a last unterminated line is dropped)."""
    with open(path, "rb") as fh:
        data = fh.read().decode("latin-1")
    parts = data.split("\n")
    lines = parts[:-1]  # the piece after the last newline is never returned
    return [ln[:-1] if ln.endswith("\r") else ln for ln in lines]


def _tokens(line: str) -> list[str]:
    t = [x for x in line.split(" ") if x]
    return t if t else [""]


class _Reader:
    def __init__(self, path: str):
        self.path = path
        self.lines = _read_lines(path)
        self.i = 0

    def line(self, what: str) -> str:
        if self.i >= len(self.lines):
            raise ValueError(f"{self.path}: unexpected end of file, expected {what}")
        ln = self.lines[self.i]
        self.i += 1
        return ln

    def tokens(self, what: str, counts=None) -> list[str]:
        t = _tokens(self.line(what))
        if counts is not None and len(t) not in counts:
            raise ValueError(f"{self.path}:{self.i}: expected {what}, found {len(t)} tokens")
        return t

    def more(self) -> bool:
        return self.i < len(self.lines)


# --------------------------------------------------------------------------
# skeleton
# --------------------------------------------------------------------------

@dataclasses.dataclass
class SkeletonFile:
    """A parsed ``Skeletool Skeleton Definition V1.0`` file (skeleton.cpp:254-530)."""
    joint_names: list[str]
    joint_type: np.ndarray      # [J] int32 (0 revolute, 1 prismatic)
    parent: np.ndarray          # [J] int32, -1 for the root
    offset: np.ndarray          # [J,3] float32
    axis: np.ndarray            # [J,3] float32 (revolute axes normalised)
    scale: np.ndarray           # [J] float32
    marker_names: list[str]
    marker_joint: np.ndarray    # [Mk] int32
    marker_offset: np.ndarray   # [Mk,3] float32
    dof_names: list[str]
    dof_limits: list            # [D] (lo, hi) or None
    dof_offsets: np.ndarray     # [D+1] int32 CSR over (dof_joint, dof_weight)
    dof_joint: np.ndarray
    dof_weight: np.ndarray

    def joint_by_name(self, name: str) -> int:
        """First joint whose name starts with ``name`` (skeleton.cpp:3655-3665), -1 if none."""
        for j, jn in enumerate(self.joint_names):
            if jn.startswith(name):
                return j
        return -1

    def last_joint_by_name(self, name: str) -> int:
        """Last joint whose name starts with ``name`` (skeleton.cpp:3667-3677), -1 if none."""
        for j in range(len(self.joint_names) - 1, -1, -1):
            if self.joint_names[j].startswith(name):
                return j
        return -1

    def bind_dofs(self) -> np.ndarray:
        """Initial dof values: zero clamped to each dof's limits (skeleton.cpp:475-482)."""
        return np.array([0.0 if lim is None else min(max(0.0, lim[0]), lim[1]) for lim in self.dof_limits],
                        np.float64)

    def children(self, j: int) -> list[int]:
        """Children in the order the loader attaches them (joint index order)."""
        return [c for c in range(len(self.joint_names)) if self.parent[c] == j]

    def base_joint(self, j: int) -> int:
        """Walk up while the joint's offset is zero (skeleton.cpp:358-361)."""
        while self.parent[j] >= 0 and not np.any(self.offset[j]):
            j = int(self.parent[j])
        return j


def load_skeleton(path: str) -> SkeletonFile:
    ext = os.path.splitext(path)[1].lower()
    if ext in (".pskel", ".bvh"):
        raise NotImplementedError(f"{path}: {ext} skeletons are not supported (only Skeletool V1.0 files)")
    r = _Reader(path)
    header = r.line("the skeleton header")
    if header != "Skeletool Skeleton Definition V1.0":
        if header in ("Skeleton v0.9", "Skeleton v0.3", "Skeleton v0.1", "Skeleton v0.10"):
            raise NotImplementedError(f"{path}: skeleton format '{header}' is not supported (only V1.0)")
        raise ValueError(f"{path}: not a skeleton file (header '{header}')")
    t = r.tokens("the number of joints", (2,))
    if t[0] != "joints:":
        raise ValueError(f"{path}: expected 'joints:'")
    nj = int(t[1])
    names, types, parents_by_name = [], [], []
    off = np.zeros((nj, 3), np.float32)
    ax = np.zeros((nj, 3), np.float32)
    sc = np.ones(nj, np.float32)
    for i in range(nj):
        t = r.tokens("joint data (10 values)", (10,))
        names.append(t[0])
        v = np.array([float(x) for x in t[3:10]], np.float32)
        off[i] = v[0:3]
        if t[1] == "revolute":
            types.append(REVOLUTE)
            a = v[3:6]
            n = np.float32(np.sqrt(np.float32(a[0] * a[0] + a[1] * a[1]) + np.float32(a[2] * a[2])))
            ax[i] = a / n if n > 0 else a
        elif t[1] == "prismatic":
            types.append(PRISMATIC)
            ax[i] = v[3:6]
        else:
            raise ValueError(f"{path}: unknown joint type '{t[1]}'")
        sc[i] = v[6]
        parents_by_name.append(t[2])
    parent = np.full(nj, -1, np.int32)
    for i in range(nj):
        # exact name match (skeleton.cpp:3643-3652); a joint whose parent is not
        # found becomes the root
        parent[i] = names.index(parents_by_name[i]) if parents_by_name[i] in names else -1
    t = r.tokens("the number of markers", (2,))
    if t[0] != "markers:":
        raise ValueError(f"{path}: expected 'markers:'")
    mnames, mjoint, moff = [], [], []
    skel = SkeletonFile(names, np.array(types, np.int32), parent, off, ax, sc, mnames, None, None, [], [], None, None,
                        None)
    for _ in range(int(t[1])):
        t = r.tokens("marker data", (6, 7, 10, 11))
        j = skel.joint_by_name(t[1])
        if j < 0:
            raise ValueError(f"{path}: unknown marker parent '{t[1]}'")
        if t[2] not in ("point", "oriented"):
            raise ValueError(f"{path}: unknown marker type '{t[2]}'")
        mnames.append(t[0])
        mjoint.append(j)
        moff.append([float(x) for x in t[3:6]])
    t = r.tokens("the number of scaling joints", (3,))
    if t[0] != "scaling" or t[1] != "joints:":
        raise ValueError(f"{path}: expected 'scaling joints:'")
    for _ in range(int(t[2])):
        t = r.tokens("scaling joint data", (2,))
        for _ in range(int(t[1])):
            r.tokens("a joint name", (1,))
    t = r.tokens("the number of dofs", (2,))
    if t[0] != "dofs:":
        raise ValueError(f"{path}: expected 'dofs:'")
    dnames, limits, doff, dj, dw = [], [], [0], [], []
    for _ in range(int(t[1])):
        t = r.tokens("dof data", (2,))
        dnames.append(t[0])
        n = int(t[1])
        lt = r.tokens("dof limits", (1, 3))
        if lt[0] == "limits" and len(lt) == 3:
            limits.append((float(np.float32(lt[1])), float(np.float32(lt[2]))))
        elif lt[0] == "nolimits" and len(lt) == 1:
            limits.append(None)
        else:
            raise ValueError(f"{path}: unknown dof limit specification")
        for _ in range(n):
            jt = r.tokens("a dof joint and weight", (2,))
            j = skel.joint_by_name(jt[0])
            if j < 0:
                raise ValueError(f"{path}: unknown joint '{jt[0]}' in dof '{dnames[-1]}'")
            dj.append(j)
            dw.append(float(jt[1]))
        doff.append(len(dj))
    skel.marker_joint = np.array(mjoint, np.int32)
    skel.marker_offset = np.array(moff, np.float32).reshape(-1, 3)
    skel.dof_names = dnames
    skel.dof_limits = limits
    skel.dof_offsets = np.array(doff, np.int32)
    skel.dof_joint = np.array(dj, np.int32)
    skel.dof_weight = np.array(dw, np.float32)
    return skel


def _axis_angle(a, th):
    c, s = math.cos(th), math.sin(th)
    x, y, z = (float(v) for v in a)
    C = 1.0 - c
    return np.array([[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                     [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                     [z * x * C - y * s, z * y * C + x * s, c + z * z * C]])


def joint_transforms(skel: SkeletonFile, dofs: np.ndarray, unit_scale: bool = False):
    """Global joint rotations [J,3,3] and translations [J,3] (joint.cpp:36-168, dof.cpp:9-17), FP64."""
    J = len(skel.joint_names)
    P = np.zeros(J)
    for d in range(len(skel.dof_names)):
        for e in range(skel.dof_offsets[d], skel.dof_offsets[d + 1]):
            P[skel.dof_joint[e]] += float(skel.dof_weight[e]) * float(dofs[d])
    R = np.zeros((J, 3, 3))
    t = np.zeros((J, 3))
    done = np.zeros(J, bool)

    def visit(j):
        if done[j]:
            return
        p = int(skel.parent[j])
        if p >= 0:
            visit(p)
        lt = skel.offset[j].astype(np.float64) * (1.0 if unit_scale else float(skel.scale[j]))
        if skel.joint_type[j] == REVOLUTE:
            lr = _axis_angle(skel.axis[j], P[j])
        else:
            lr = np.eye(3)
            lt = lt + skel.axis[j].astype(np.float64) * P[j]
        R[j] = R[p] @ lr if p >= 0 else lr
        t[j] = R[p] @ lt + t[p] if p >= 0 else lt
        done[j] = True

    for j in range(J):
        visit(j)
    return R, t


def marker_positions(skel: SkeletonFile) -> np.ndarray:
    """Global marker positions at the bind dofs with the joint scales (marker.cpp:83-88; unscaled offsets)."""
    R, t = joint_transforms(skel, skel.bind_dofs())
    out = np.zeros((len(skel.marker_names), 3))
    for m, j in enumerate(skel.marker_joint):
        out[m] = R[j] @ skel.marker_offset[m].astype(np.float64) + t[j]
    return out.astype(np.float32)


# --------------------------------------------------------------------------
# meshes
# --------------------------------------------------------------------------

@dataclasses.dataclass
class Mesh:
    """A triangle mesh read from ``.obj`` (trimesh.cpp:337-480)."""
    vertices: np.ndarray        # [N,3] float32
    faces: np.ndarray           # [F,3] int32
    normals: np.ndarray         # [N,3] float32, area-weighted and normalised
    colors: np.ndarray          # [N,3] float32 (white where the file has none)
    texcoords: np.ndarray       # [T,2] float32
    face_tindex: np.ndarray | None  # [F,3] int32, None when no face has texture indices

    def face_uvs(self) -> np.ndarray:
        """Per-face-corner UVs [F*6] (the renderer's ``texture_coordinates`` attribute)."""
        if self.face_tindex is None:
            raise ValueError("the mesh has no texture coordinates")
        return self.texcoords[self.face_tindex].reshape(-1).astype(np.float32)


def vertex_normals(vertices: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """Sum of face cross products in reverse face order, then normalised, in FP32 (trimesh.cpp:838-857)."""
    v = np.asarray(vertices, np.float32)
    f = np.asarray(faces, np.int64)[::-1]
    a = v[f[:, 1]] - v[f[:, 0]]
    b = v[f[:, 2]] - v[f[:, 0]]
    fn = np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1], a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                   a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1).astype(np.float32)
    n = np.zeros_like(v)
    # corners interleaved face by face, so every vertex sums its faces in the reference's order
    np.add.at(n, f.reshape(-1), np.repeat(fn, 3, axis=0))
    sq = (n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2]
    ln = np.sqrt(sq)
    ok = sq > 0
    n[ok] = n[ok] / ln[ok, None]
    return n


def load_obj(path: str) -> Mesh:
    if os.path.splitext(path)[1] != ".obj":
        raise NotImplementedError(f"{path}: only .obj meshes are supported")
    verts, cols, tex, faces, tidx = [], {}, [], [], []
    all_t = True
    for ln in _read_lines(path):
        t = _tokens(ln)
        k = t[0]
        if k == "v":
            verts.append([float(x) for x in t[1:4]])
            if len(t) > 5:
                cols[len(verts) - 1] = [float(x) for x in t[4:7]]
        elif k == "vt":
            tex.append([float(x) for x in t[1:3]])
        elif k == "f":
            vi, ti = [], []
            for tok in t[1:]:
                sub = tok.split("/")
                vi.append(int(sub[0]) - 1)
                if len(sub) > 1 and sub[1]:
                    ti.append(int(sub[1]) - 1)
            for d in range(2, len(vi)):
                faces.append([vi[0], vi[d - 1], vi[d]])
                if len(ti) == len(vi):
                    tidx.append([ti[0], ti[d - 1], ti[d]])
                else:
                    all_t = False
                    tidx.append([0, 0, 0])
    v = np.array(verts, np.float32).reshape(-1, 3)
    f = np.array(faces, np.int64).reshape(-1, 3)
    if f.size and (f.min() < 0 or f.max() >= v.shape[0]):
        raise ValueError(f"{path}: vertex index out of range")
    c = np.ones_like(v)
    for i, rgb in cols.items():
        c[i] = rgb
    ftex = np.array(tidx, np.int32).reshape(-1, 3) if (tex and all_t and faces) else None
    return Mesh(v, f.astype(np.int32), vertex_normals(v, f), c, np.array(tex, np.float32).reshape(-1, 2), ftex)


_SEGMENT_WEIGHT = {}
for _ids, _w in (((0, 6, 7, 10, 12, 5), 10.0), ((9,), 15.0), ((11, 8), 50.0),
                 ((14, 15, 16, 17, 18, 19, 1, 3, 4, 2, 13), 200.0)):
    for _i in _ids:
        _SEGMENT_WEIGHT[_i] = _w


def segmentation_weights(mesh_path: str, n_vertices: int) -> np.ndarray:
    """Per-vertex rigidity weights from ``segmentation.txt`` beside the mesh (trimesh.cpp:1305-1380); 1 without it."""
    p = os.path.join(os.path.dirname(mesh_path), "segmentation.txt")
    if not os.path.exists(p):
        return np.ones(n_vertices, np.float32)
    with open(p) as fh:
        rows = fh.read().split("\n")
    if len(rows) < n_vertices:
        raise ValueError(f"{p}: {len(rows)} lines for {n_vertices} vertices")
    w = np.empty(n_vertices, np.float32)
    for v in range(n_vertices):
        seg = int(rows[v].strip())
        if seg not in _SEGMENT_WEIGHT:
            raise ValueError(f"{p}: vertex {v}: no segmentation category {seg}")
        w[v] = _SEGMENT_WEIGHT[seg]
    return w


# --------------------------------------------------------------------------
# skin and character
# --------------------------------------------------------------------------

def load_skin(path: str, skel: SkeletonFile):
    """``.skin`` file -> (skinning joint per bone [S], per-vertex [(bone, weight), ...])
    (skinnedcharacter.cpp:149-206)."""
    ext = os.path.splitext(path)[1]
    if ext != ".skin":
        raise NotImplementedError(f"{path}: only .skin skinning files are supported")
    r = _Reader(path)
    if r.line("the skin header") != "Skeletool character skinning file V1.0":
        raise ValueError(f"{path}: not a skin file")
    if r.line("'bones:'") != "bones:":
        raise ValueError(f"{path}: expected 'bones:'")
    bones = r.tokens("the bone names")
    sj = []
    for b in bones:
        j = skel.last_joint_by_name(b)
        if j < 0:
            raise ValueError(f"{path}: bone '{b}' matches no joint")
        sj.append(j)
    if r.line("'vertex weights:'") != "vertex weights:":
        raise ValueError(f"{path}: expected 'vertex weights:'")
    per_vertex = []
    while r.more():
        t = _tokens(r.line("vertex weights"))
        per_vertex.append([(int(t[j]), float(np.float32(t[j + 1]))) for j in range(1, len(t) - 1, 2)])
    return np.array(sj, np.int32), per_vertex


@dataclasses.dataclass
class CharacterFile:
    """A loaded ``.character`` file: skeleton, base mesh and skinning."""
    path: str
    skeleton: SkeletonFile
    mesh_path: str
    mesh: Mesh
    skin_joint: np.ndarray          # [S] int32
    skin_index: np.ndarray          # [N,K] int32
    skin_weight: np.ndarray         # [N,K] float32

    def skin_scale(self) -> np.ndarray:
        """Scale of each skinning joint's transform (DQSkinningGPUOp.cpp:271-281):
        the first child's scale, else the scale of the joint's base."""
        sk = self.skeleton
        out = np.empty(len(self.skin_joint), np.float32)
        for s, j in enumerate(self.skin_joint):
            ch = sk.children(int(j))
            out[s] = sk.scale[ch[0]] if ch else sk.scale[sk.base_joint(int(j))]
        return out

    def character(self) -> Character:
        """The arrays ``SkinningEngine`` takes (joints must be listed after their parents)."""
        sk = self.skeleton
        for j, p in enumerate(sk.parent):
            if p >= j:
                raise ValueError(f"{self.path}: joint '{sk.joint_names[j]}' is listed before its parent; "
                                 "the device forward kinematics needs parents first")
        return Character(sk.parent.copy(), sk.joint_type.copy(), sk.offset.copy(), sk.axis.copy(),
                         sk.dof_offsets.copy(), sk.dof_joint.copy(), sk.dof_weight.copy(), self.skin_joint.copy(),
                         self.mesh.vertices.copy(), self.mesh.normals.copy(), self.skin_index.copy(),
                         joint_scale=sk.scale.copy(), skin_scale=self.skin_scale())


def load_character(path: str) -> CharacterFile:
    r = _Reader(path)
    header = r.line("the character header")
    if header != "skeletool character file v1.0":
        if header in ("skeletool character file v0.3", "skeletool character file v0.1"):
            raise NotImplementedError(f"{path}: character format '{header}' (separate .dof file) is not supported")
        raise ValueError(f"{path}: not a character file (header '{header}')")
    base = os.path.dirname(path)
    files = {}
    while r.more():
        t = _tokens(r.line("a section"))
        if t[0] in ("skeleton", "mesh", "skin", "pose"):
            files[t[0]] = os.path.join(base, _tokens(r.line(f"the {t[0]} path"))[0])
    if "pose" in files:
        raise NotImplementedError(f"{path}: initial-pose files are not supported")
    for k in ("skeleton", "mesh", "skin"):
        if k not in files:
            raise ValueError(f"{path}: no {k} path")
    skel = load_skeleton(files["skeleton"])
    mesh = load_obj(files["mesh"])
    sj, per_vertex = load_skin(files["skin"], skel)
    N = mesh.vertices.shape[0]
    if len(per_vertex) < N:
        raise ValueError(f"{files['skin']}: {len(per_vertex)} weight rows for {N} vertices")
    per_vertex = per_vertex[:N]  # the ops read the rows of the mesh's vertices only
    K = len(per_vertex[0]) if per_vertex else 0
    if K == 0 or any(len(x) != K for x in per_vertex):
        raise ValueError(f"{files['skin']}: every vertex needs the same number of weights")
    idx = np.array([[b for b, _ in x] for x in per_vertex], np.int32)
    w = np.array([[wt for _, wt in x] for x in per_vertex], np.float32)
    if idx.min() < 0 or idx.max() >= len(sj):
        raise ValueError(f"{files['skin']}: bone index out of range")
    return CharacterFile(path, skel, files["mesh"], mesh, sj, idx, w)


# --------------------------------------------------------------------------
# embedded graph
# --------------------------------------------------------------------------

def _neighbours(n_vertices: int, faces: np.ndarray):
    """Sorted vertex neighbours from the faces (trimesh.cpp:896-911) as a CSR matrix."""
    import scipy.sparse as sp
    f = np.asarray(faces, np.int64)
    r = np.concatenate([f[:, 0], f[:, 0], f[:, 1], f[:, 1], f[:, 2], f[:, 2]])
    c = np.concatenate([f[:, 1], f[:, 2], f[:, 0], f[:, 2], f[:, 0], f[:, 1]])
    a = sp.csr_matrix((np.ones(r.shape[0], np.int8), (r, c)), shape=(n_vertices, n_vertices))
    a.sum_duplicates()
    a.sort_indices()
    return a


def _hops(adj, sources) -> np.ndarray:
    """Breadth-first hop distances [len(sources), N] (trimesh.cpp:868-890), unreached = 1000000."""
    from scipy.sparse.csgraph import shortest_path
    d = shortest_path(adj, method="D", unweighted=True, indices=np.asarray(sources, np.int64))
    d = np.atleast_2d(d)
    out = np.full(d.shape, _UNREACHED, np.int64)
    ok = np.isfinite(d)
    out[ok] = d[ok].astype(np.int64)
    return out


def _extreme_y(v: np.ndarray):
    """First vertex with the largest and with the smallest y (EmbeddedGraph.cpp:48-62)."""
    y = v[:, 1]
    hi = lo = -1
    maxy, miny = np.float32(-10000.0), np.float32(100000.0)
    for i in range(v.shape[0]):
        if y[i] > maxy:
            maxy, hi = y[i], i
        if y[i] < miny:
            miny, lo = y[i], i
    if hi < 0 or lo < 0:
        raise ValueError("mesh y range outside (-10000, 100000)")
    return hi, lo


@dataclasses.dataclass
class GraphFile:
    """An embedded graph built from a character and a graph mesh (EmbeddedGraph.cpp:5-490)."""
    eg: EGData                  # arrays for ``EmbeddedGraphEngine``
    n2n_offsets: np.ndarray     # [M] node neighbours (graph-mesh edges, ascending)
    n2n_sizes: np.ndarray
    n2n_indices: np.ndarray
    rigidity: np.ndarray        # [M] float32
    radius: np.ndarray          # [M] int hop radius of every node

    @property
    def max_connections(self) -> int:
        return int(self.n2n_sizes.max())


def load_graph(character: CharacterFile, graph_mesh_path: str, refinement: bool = False) -> GraphFile:
    mesh = character.mesh
    gm = load_obj(graph_mesh_path)
    V = mesh.vertices
    G = gm.vertices
    N, M = V.shape[0], G.shape[0]
    adj = _neighbours(N, mesh.faces)
    gadj = _neighbours(M, gm.faces)
    hi, lo = _extreme_y(V)
    ghi, glo = _extreme_y(G)
    dh = _hops(adj, [hi, lo])
    dg = _hops(gadj, [ghi, glo])
    mesh_hi, mesh_lo = dh[0] != _UNREACHED, dh[1] != _UNREACHED
    # nodes: the closest unused vertex in the same connected parts (EmbeddedGraph.cpp:120-155)
    used = np.zeros(N, bool)
    node_vertex = np.empty(M, np.int32)
    for n in range(M):
        if gadj.indptr[n + 1] == gadj.indptr[n]:
            raise ValueError(f"{graph_mesh_path}: graph vertex {n} has no neighbour")
        d = V - G[n]
        dist = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        ok = (~used) & (mesh_hi == (dg[0, n] != _UNREACHED)) & (mesh_lo == (dg[1, n] != _UNREACHED))
        ok &= dist < np.float32(np.finfo(np.float32).max)
        if not ok.any():
            raise ValueError(f"{graph_mesh_path}: no free mesh vertex for graph vertex {n}")
        cand = np.where(ok, dist, np.inf)
        v = int(np.argmin(cand))
        used[v] = True
        node_vertex[n] = v
    n2n_sizes = np.diff(gadj.indptr).astype(np.int32)
    n2n_offsets = gadj.indptr[:-1].astype(np.int32)
    n2n_indices = gadj.indices.astype(np.int32)
    # radius: half the largest hop distance to a graph neighbour's vertex, at
    # least 3 (:218-238); connections (:240-280): Gaussian of hop distance /
    # radius inside the radius, else the nearest node (the last one at the
    # smallest distance) with weight 1.  Hop distances are taken for a chunk of
    # nodes at a time so that only [chunk, N] is held.
    radius = np.empty(M, np.int64)
    pair_node, pair_vertex, pair_w = [], [], []
    best = np.full(N, np.inf)
    best_node = np.full(N, -1, np.int64)
    for c0 in range(0, M, 64):
        nodes = np.arange(c0, min(M, c0 + 64))
        dist = _hops(adj, node_vertex[nodes])  # [c, N]
        for q, n in enumerate(nodes):
            nb = n2n_indices[n2n_offsets[n]:n2n_offsets[n] + n2n_sizes[n]]
            radius[n] = max(max(0, int(dist[q, node_vertex[nb]].max())) // 2, 3)
        dn = dist.astype(np.float32) / radius[nodes].astype(np.float32)[:, None]
        qi, vi = np.nonzero(dn <= np.float32(1.0))
        pair_node.append(nodes[qi])
        pair_vertex.append(vi)
        pair_w.append(np.exp(-0.5 * dn[qi, vi].astype(np.float64) ** 2).astype(np.float32))
        df = dist.astype(np.float32)
        cmin = df.min(axis=0)
        clast = nodes[len(nodes) - 1 - np.argmin(df[::-1], axis=0)]
        upd = cmin <= best
        best[upd] = cmin[upd]
        best_node[upd] = clast[upd]
    pn = np.concatenate(pair_node)
    pv = np.concatenate(pair_vertex)
    pw = np.concatenate(pair_w)
    lonely = np.setdiff1d(np.arange(N), pv)
    pn = np.concatenate([pn, best_node[lonely]])
    pv = np.concatenate([pv, lonely])
    pw = np.concatenate([pw, np.ones(lonely.size, np.float32)])
    order = np.lexsort((pn, pv))  # by vertex, then node: the reference's connection order
    pn, pv, pw = pn[order], pv[order], pw[order]
    # normalisation: FP32 sum in node order, then one division each (:304-321)
    wsum = np.zeros(N, np.float32)
    np.add.at(wsum, pv, pw)
    v2n_indices = pn.astype(np.int32)
    v2n_weights = (pw / wsum[pv]).astype(np.float32)
    sizes = np.bincount(pv, minlength=N).astype(np.int32)
    v2n_offsets = np.zeros(N, np.int32)
    v2n_offsets[1:] = np.cumsum(sizes)[:-1]
    # node -> vertex lists: vertices ascending (:385-410)
    owner = np.repeat(np.arange(N), sizes)
    order = np.lexsort((owner, v2n_indices))
    n2v_indices = owner[order].astype(np.int32)
    n2v_weights = v2n_weights[order]
    n2v_sizes = np.bincount(v2n_indices, minlength=M).astype(np.int32)
    n2v_offsets = np.zeros(M, np.int32)
    n2v_offsets[1:] = np.cumsum(n2v_sizes)[:-1]
    # rigidity: mean segmentation weight over each node's vertex connections (:460-490)
    seg = segmentation_weights(character.mesh_path, N)
    contrib = seg[owner]
    if refinement:
        contrib = np.where(contrib < np.float32(20.0), contrib / np.float32(10.0), contrib).astype(np.float32)
    rig = np.zeros(M, np.float32)
    np.add.at(rig, v2n_indices[order], contrib[order])  # each node sums its vertices in ascending order
    rig = (rig / n2v_sizes.astype(np.float32)).astype(np.float32)
    # markers: nearest node by base-vertex distance (:503-531)
    mk = marker_positions(character.skeleton)
    nodes_pos = V[node_vertex]
    marker_node = np.empty(mk.shape[0], np.int32)
    for m in range(mk.shape[0]):
        d = nodes_pos - mk[m]
        marker_node[m] = int(np.argmin(np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])))
    eg = EGData(V.copy(), mesh.faces.copy(), node_vertex, v2n_offsets, sizes, v2n_indices, v2n_weights, n2v_offsets,
                n2v_sizes, n2v_indices, n2v_weights, mk if mk.shape[0] else None,
                marker_node if mk.shape[0] else None)
    return GraphFile(eg, n2n_offsets, n2n_sizes, n2n_indices, rig, radius.astype(np.int32))
