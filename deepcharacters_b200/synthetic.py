"""Seeded synthetic scenes for the deform-and-render chain.

The reference trains on captured multi-view video with character, skin and
graph files that are not part of this project.  Everything here builds
stand-ins with the same shapes and value ranges, in millimetres, because the
reference ray test divides coordinates by 1000 and rejects unit-scale meshes
(CudaRenderer/cpp/src/Utils/RendererUtil.h:29-50):

* icospheres of radius 1000 with per-vertex jitter,
* pinhole cameras (row-major 3x4 world->camera extrinsics, 3x3 intrinsics,
  camera +z forward, +y down), as consumed by ``CudaRendererGpu``
  (CudaRenderer/cpp/src/TensorflowOperators/CudaRenderer/CudaRenderer.cpp:332-333),
* a random kinematic tree of revolute joints (three per skeletal joint),
* per-vertex skinning weights on the K nearest joints,
* an embedded graph (farthest-point nodes, K nearest nodes per vertex with
  normalised inverse-distance weights) in the CSR layout of
  Skeletool/Mesh/EmbeddedGraph.cpp:379-548,
* distance-transform images in the uint8 encoding that
  MultiViewSilhouetteLossGPUOp.cu:62-63 decodes.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

MM = 1000.0  # one metre in reference units


def rng_for(seed: int, sub: int | None = None) -> np.random.Generator:
    """PCG64 stream for a configuration seed; ``sub`` selects a per-frame stream."""
    s = seed if sub is None else seed * 1000 + sub
    return np.random.Generator(np.random.PCG64(s))


def frame_rng(seed: int, frame: int) -> np.random.Generator:
    """Stream of one frame's per-frame inputs (node deltas, colours, lighting,
    targets): a frame's data depends only on (seed, frame), so the frames a
    data-parallel rank generates for itself equal its slice of the whole job."""
    return np.random.Generator(np.random.PCG64(np.random.SeedSequence([int(seed), 1 + int(frame)])))


# ----------------------------------------------------------------------------
# meshes
# ----------------------------------------------------------------------------

def icosphere(subdiv: int) -> tuple[np.ndarray, np.ndarray]:
    """Unit icosphere: ``10*4**subdiv + 2`` vertices, ``20*4**subdiv`` faces.

    Faces are wound counter-clockwise seen from outside (outward normals for
    ``cross(v1 - v0, v2 - v0)``)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    for _ in range(subdiv):
        nv = v.shape[0]
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], axis=0)
        key = np.minimum(e[:, 0], e[:, 1]) * (nv + 1) + np.maximum(e[:, 0], e[:, 1])
        uniq, inv = np.unique(key, return_inverse=True)
        a = uniq // (nv + 1)
        b = uniq % (nv + 1)
        mid = v[a] + v[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        mid_id = nv + inv
        nf = f.shape[0]
        m01, m12, m20 = mid_id[:nf], mid_id[nf:2 * nf], mid_id[2 * nf:]
        f = np.concatenate([
            np.stack([f[:, 0], m01, m20], 1),
            np.stack([f[:, 1], m12, m01], 1),
            np.stack([f[:, 2], m20, m12], 1),
            np.stack([m01, m12, m20], 1)], axis=0)
        v = np.concatenate([v, mid], axis=0)
    return v, f.astype(np.int32)


def sphere_mesh(subdiv: int, rng: np.random.Generator, radius: float = MM,
                jitter: float = 0.01 * MM) -> tuple[np.ndarray, np.ndarray]:
    """Icosphere of ``radius`` mm with N(0, jitter) per-coordinate jitter (float32)."""
    v, f = icosphere(subdiv)
    v = v * radius + rng.normal(0.0, jitter, size=v.shape)
    return v.astype(np.float32), f


def spherical_uvs(verts: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """Per-face-corner UVs ``[F*6]`` from a spherical projection.

    The seam is handled per face: corners whose longitude wraps are shifted so
    a face never spans the whole texture."""
    p = verts.astype(np.float64)
    p = p / np.linalg.norm(p, axis=1, keepdims=True)
    u = 0.5 + np.arctan2(p[:, 0], p[:, 2]) / (2 * np.pi)
    v = 0.5 - np.arcsin(np.clip(p[:, 1], -1, 1)) / np.pi
    fu = u[faces]
    fv = v[faces]
    span = fu.max(1) - fu.min(1)
    wrap = span > 0.5
    fu[wrap] = np.where(fu[wrap] < 0.5, fu[wrap] + 1.0, fu[wrap])
    fu = np.clip(fu, 0.0, 1.0)
    uv = np.stack([fu, 1.0 - fv], axis=2)  # reference flips V again when sampling
    return uv.reshape(-1).astype(np.float32)


def vertex_faces_csr(n_verts: int, faces: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Vertex->incident-face CSR with faces in increasing index order.

    Same content and order as CUDABasedRasterization::getVertexFaces
    (CudaRenderer/cpp/src/Renderer/CUDABasedRasterization.cpp:154-183):
    returns ``vertex_faces[int]`` and ``vertex_faces_id[N,2] = (start, count)``."""
    fid = np.repeat(np.arange(faces.shape[0], dtype=np.int64), 3)
    vid = faces.reshape(-1).astype(np.int64)
    order = np.lexsort((fid, vid))
    vf = fid[order].astype(np.int32)
    counts = np.bincount(vid, minlength=n_verts).astype(np.int32)
    starts = np.zeros(n_verts, dtype=np.int32)
    starts[1:] = np.cumsum(counts)[:-1]
    return vf, np.stack([starts, counts], 1).astype(np.int32)


# ----------------------------------------------------------------------------
# cameras
# ----------------------------------------------------------------------------

def look_at(position, target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """Row-major 3x4 world->camera matrix; camera +z looks at ``target``, +y is down."""
    c = np.asarray(position, np.float64)
    z = np.asarray(target, np.float64) - c
    z /= np.linalg.norm(z)
    y = -np.asarray(up, np.float64)
    y = y - z * np.dot(y, z)
    y /= np.linalg.norm(y)
    x = np.cross(y, z)
    r = np.stack([x, y, z], 0)
    return np.concatenate([r, (-r @ c)[:, None]], 1)


def intrinsics(fx: float, fy: float, cx: float, cy: float) -> np.ndarray:
    return np.array([[fx, 0, cx], [0, fy, cy], [0, 0, 1]], np.float64)


def camera_ring(n_views: int, radius: float, fx: float, width: int, height: int,
                start_angle: float = 0.0) -> tuple[np.ndarray, np.ndarray]:
    """``n_views`` cameras on a ring in the xz-plane looking at the origin.

    Returns extrinsics ``[n_views*12]`` and intrinsics ``[n_views*9]`` (float32),
    the per-frame layout of the renderer op (``[B, 12C]`` / ``[B, 9C]``)."""
    ex, ins = [], []
    for i in range(n_views):
        a = start_angle + 2.0 * math.pi * i / n_views
        ex.append(look_at((radius * math.sin(a), 0.0, radius * math.cos(a))))
        ins.append(intrinsics(fx, fx, width / 2.0, height / 2.0))
    return (np.concatenate([e.reshape(-1) for e in ex]).astype(np.float32),
            np.concatenate([k.reshape(-1) for k in ins]).astype(np.float32))


# ----------------------------------------------------------------------------
# kinematic tree and skinning
# ----------------------------------------------------------------------------

@dataclasses.dataclass
class Skeleton:
    """Revolute-joint kinematic tree in the reference's joint model.

    Every skeletal joint is three revolute joints about the local x, y and z
    axes with zero offset between them (Skeletool/Character/joint.cpp:144-148),
    so ``n_joints = 3 * n_skel``.  Joint ``j`` has parent ``parent[j]`` (-1 for
    the root), local offset ``offset[j]`` (mm) and unit axis ``axis[j]``; each DOF
    drives exactly one joint with weight 1 (Skeletool/Character/dof.cpp:9-17).
    Skinning joint ``s`` is the last revolute joint of skeletal joint ``s``."""
    parent: np.ndarray      # [J] int32
    offset: np.ndarray      # [J,3] float32
    axis: np.ndarray        # [J,3] float32
    dof_joint: np.ndarray   # [D] int32: joint driven by each dof
    dof_weight: np.ndarray  # [D] float32
    skin_joint: np.ndarray  # [S] int32: joint index of each skinning joint
    scale: float = 1.0

    @property
    def n_joints(self) -> int:
        return int(self.parent.shape[0])

    @property
    def n_dofs(self) -> int:
        return int(self.dof_joint.shape[0])

    @property
    def n_skin(self) -> int:
        return int(self.skin_joint.shape[0])


def random_skeleton(n_skel: int, rng: np.random.Generator, radius: float = MM) -> Skeleton:
    """Random tree: parent uniform over earlier joints, positions inside the sphere."""
    pos = np.zeros((n_skel, 3))
    par = np.full(n_skel, -1, np.int64)
    for j in range(1, n_skel):
        par[j] = rng.integers(0, j)
        while True:
            p = rng.uniform(-0.8 * radius, 0.8 * radius, 3)
            if np.linalg.norm(p) < 0.8 * radius:
                break
        pos[j] = p
    J = 3 * n_skel
    parent = np.full(J, -1, np.int32)
    offset = np.zeros((J, 3), np.float32)
    axis = np.zeros((J, 3), np.float32)
    for j in range(n_skel):
        base = 3 * j
        if par[j] >= 0:
            parent[base] = 3 * par[j] + 2
            offset[base] = pos[j] - pos[par[j]]
        else:
            offset[base] = pos[j]
        parent[base + 1] = base
        parent[base + 2] = base + 1
        axis[base + 0] = (1, 0, 0)
        axis[base + 1] = (0, 1, 0)
        axis[base + 2] = (0, 0, 1)
    dof_joint = np.arange(J, dtype=np.int32)
    dof_weight = np.ones(J, np.float32)
    skin_joint = (3 * np.arange(n_skel) + 2).astype(np.int32)
    return Skeleton(parent, offset, axis, dof_joint, dof_weight, skin_joint)


def rest_joint_positions(sk: Skeleton) -> np.ndarray:
    """Global joint positions at zero pose."""
    p = np.zeros((sk.n_joints, 3))
    for j in range(sk.n_joints):
        base = p[sk.parent[j]] if sk.parent[j] >= 0 else 0.0
        p[j] = base + sk.offset[j] * sk.scale
    return p


def skinning_weights(verts: np.ndarray, sk: Skeleton, k: int, rng: np.random.Generator, smooth: bool = False):
    """Per vertex the ``k`` nearest skinning joints (Euclidean, rest pose) with
    Dirichlet(1) weights, or with ``smooth`` weights that are continuous over
    the surface (neighbouring vertices get nearly equal blends, so large joint
    angles fold the surface instead of tearing it).
    Returns ``(indices[N,k] int32, weights[N,k] float32)``."""
    jp = rest_joint_positions(sk)[sk.skin_joint]
    d = np.linalg.norm(verts[:, None, :].astype(np.float64) - jp[None], axis=2)
    idx = np.argsort(d, axis=1, kind="stable")[:, :k].astype(np.int32)
    if smooth:
        # w_k proportional to (distance of the (k+1)-th nearest joint - own
        # distance): a joint's weight falls to zero exactly where it leaves
        # the k nearest, so the weights are continuous over the surface
        order = np.argsort(d, axis=1, kind="stable")
        dk = np.take_along_axis(d, order[:, :k + 1], axis=1)
        w = dk[:, k:k + 1] - dk[:, :k] + 1e-6
        w = (w / w.sum(axis=1, keepdims=True)).astype(np.float32)
    else:
        w = rng.dirichlet(np.ones(k), size=verts.shape[0]).astype(np.float32)
    return idx, w


def random_pose(sk: Skeleton, rng: np.random.Generator, amplitude: float = 0.5) -> np.ndarray:
    return rng.uniform(-amplitude, amplitude, sk.n_dofs).astype(np.float32)


# ----------------------------------------------------------------------------
# embedded graph
# ----------------------------------------------------------------------------

@dataclasses.dataclass
class EmbeddedGraph:
    """Embedded deformation graph in the reference's CSR layout.

    ``node_vertex[n]``: base-mesh vertex the node sits on.  Vertex->node CSR:
    ``v2n_offsets/sizes/indices/weights``.  Node->vertex CSR (same weights, for
    the gather-form backward): ``n2v_offsets/sizes/indices/weights``."""
    node_vertex: np.ndarray
    v2n_offsets: np.ndarray
    v2n_sizes: np.ndarray
    v2n_indices: np.ndarray
    v2n_weights: np.ndarray
    n2v_offsets: np.ndarray
    n2v_sizes: np.ndarray
    n2v_indices: np.ndarray
    n2v_weights: np.ndarray

    @property
    def n_nodes(self) -> int:
        return int(self.node_vertex.shape[0])


def farthest_point_sample(verts: np.ndarray, n: int, rng: np.random.Generator) -> np.ndarray:
    p = verts.astype(np.float64)
    sel = np.empty(n, np.int64)
    sel[0] = rng.integers(0, p.shape[0])
    d = np.linalg.norm(p - p[sel[0]], axis=1)
    for i in range(1, n):
        sel[i] = int(np.argmax(d))
        d = np.minimum(d, np.linalg.norm(p - p[sel[i]], axis=1))
    return sel


def embedded_graph(verts: np.ndarray, n_nodes: int, k: int, rng: np.random.Generator) -> EmbeddedGraph:
    node_vertex = farthest_point_sample(verts, n_nodes, rng)
    g = verts[node_vertex].astype(np.float64)
    N = verts.shape[0]
    idx = np.empty((N, k), np.int64)
    dist = np.empty((N, k))
    chunk = 8192
    for s in range(0, N, chunk):
        d = np.linalg.norm(verts[s:s + chunk, None, :].astype(np.float64) - g[None], axis=2)
        o = np.argsort(d, axis=1, kind="stable")[:, :k]
        idx[s:s + chunk] = o
        dist[s:s + chunk] = np.take_along_axis(d, o, 1)
    w = 1.0 / np.maximum(dist, 1e-3)
    w /= w.sum(1, keepdims=True)
    v2n_sizes = np.full(N, k, np.int32)
    v2n_offsets = (np.arange(N) * k).astype(np.int32)
    v2n_indices = idx.reshape(-1).astype(np.int32)
    v2n_weights = w.reshape(-1).astype(np.float32)
    vid = np.repeat(np.arange(N), k)
    order = np.lexsort((vid, v2n_indices))
    n2v_indices = vid[order].astype(np.int32)
    n2v_weights = v2n_weights[order]
    n2v_sizes = np.bincount(v2n_indices, minlength=n_nodes).astype(np.int32)
    n2v_offsets = np.zeros(n_nodes, np.int32)
    n2v_offsets[1:] = np.cumsum(n2v_sizes)[:-1]
    return EmbeddedGraph(node_vertex.astype(np.int32), v2n_offsets, v2n_sizes, v2n_indices,
                         v2n_weights, n2v_offsets, n2v_sizes, n2v_indices, n2v_weights)


# ----------------------------------------------------------------------------
# images
# ----------------------------------------------------------------------------

def ellipse_mask(width: int, height: int, rng: np.random.Generator) -> np.ndarray:
    """Random filled ellipse (bool ``[H,W]``): centre +-64 px, semi-axes U[80,200]."""
    cx = width / 2 + rng.uniform(-64, 64)
    cy = height / 2 + rng.uniform(-64, 64)
    a = rng.uniform(80, 200)
    b = rng.uniform(80, 200)
    th = rng.uniform(0, np.pi)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    x = xx + 0.5 - cx
    y = yy + 0.5 - cy
    c, s = math.cos(th), math.sin(th)
    u = (c * x + s * y) / a
    v = (-s * x + c * y) / b
    return (u * u + v * v) <= 1.0


def exact_edt(mask: np.ndarray) -> np.ndarray:
    """Euclidean distance from every pixel to the nearest ``True`` pixel (exact EDT)."""
    from scipy import ndimage
    return ndimage.distance_transform_edt(~mask.astype(bool))


def encode_dt(mask: np.ndarray) -> np.ndarray:
    """Distance-transform image in the reference's uint8 encoding.

    The reference only decodes these images (MultiViewSilhouetteLossGPUOp.cu:62-63:
    ``v >= 127 -> (v - 127) * 2``; ``v <= 127`` is foreground; ``127`` marks the
    silhouette boundary, :163).  The encoder that wrote its training data is not
    part of the reference, so this one follows what the decoder implies:
    boundary pixels (foreground with a 4-neighbour in the background) are 127,
    other foreground pixels hold ``min(d_out, 126)`` with ``d_out`` the distance to
    the background, background pixels hold ``127 + min(ceil(d_in / 2), 128)``
    with ``d_in`` the distance to the foreground."""
    m = mask.astype(bool)
    pad = np.pad(m, 1, constant_values=False)
    interior = pad[1:-1, 1:-1] & pad[:-2, 1:-1] & pad[2:, 1:-1] & pad[1:-1, :-2] & pad[1:-1, 2:]
    boundary = m & ~interior
    d_in = exact_edt(m)        # background -> nearest foreground
    d_out = exact_edt(~m)      # foreground -> nearest background
    out = np.empty(m.shape, np.uint8)
    out[m] = np.minimum(np.round(d_out[m]), 126).astype(np.uint8)
    out[~m] = (127 + np.minimum(np.ceil(d_in[~m] / 2.0), 128)).astype(np.uint8)
    out[boundary] = 127
    return out


def dt_image(width: int, height: int, rng: np.random.Generator) -> np.ndarray:
    """uint8 ``[H,W]`` distance-transform image of a random ellipse (stored row-major,
    ``y * W + x``, as MultiViewSilhouetteLossGPUOp.cu:62 indexes it)."""
    return encode_dt(ellipse_mask(width, height, rng))


# ----------------------------------------------------------------------------
# render scenes
# ----------------------------------------------------------------------------

def sh_coefficients(n: int, rng: np.random.Generator) -> np.ndarray:
    """Plausible second-order SH lighting ``[n, 27]``: ambient ~1, small bands."""
    sh = rng.normal(0.0, 0.1, size=(n, 27)).astype(np.float32)
    sh[:, 0] = 1.0
    sh[:, 9] = 1.0
    sh[:, 18] = 1.0
    return sh


def render_scene(subdiv: int, batch: int, views: int, width: int, height: int, seed: int,
                 fx: float | None = None, ring_radius: float = 3.0 * MM, texture_size: int = 64,
                 per_frame_jitter: bool = True) -> dict:
    """Inputs of one ``CudaRendererGpu`` call on a jittered icosphere.

    Cameras sit on a ring in the xz-plane (the first one at (0,0,ring_radius))
    looking at the origin; ``fx`` defaults to ``600 * min(W, H) / 512``.  Each
    frame re-jitters the vertices (independent per-frame stream) so frames
    differ.  Returns numpy arrays in the op's layouts."""
    rng = rng_for(seed)
    v_unit, faces = icosphere(subdiv)
    N = v_unit.shape[0]
    verts = np.empty((batch, N, 3), np.float32)
    for b in range(batch):
        r = rng_for(seed, b) if per_frame_jitter else rng_for(seed)
        verts[b] = (v_unit * MM + r.normal(0.0, 0.01 * MM, size=v_unit.shape)).astype(np.float32)
    if fx is None:
        fx = 600.0 * min(width, height) / 512.0
    ex, it = camera_ring(views, ring_radius, fx, width, height)
    colors = rng.uniform(0.0, 1.0, size=(batch, N, 3)).astype(np.float32)
    texture = rng.uniform(0.0, 1.0, size=(batch, texture_size, texture_size, 3)).astype(np.float32)
    sh = sh_coefficients(batch * views, rng).reshape(batch, views, 27)
    target = rng.uniform(0.0, 1.0, size=(batch, views, height, width, 3)).astype(np.float32)
    return dict(faces=faces, verts=verts, colors=colors, texture=texture, sh=sh,
                extr=np.tile(ex[None], (batch, 1)), intr=np.tile(it[None], (batch, 1)),
                texcoords=spherical_uvs(verts[0], faces), target=target,
                N=N, F=faces.shape[0], B=batch, C=views, W=width, H=height)


@dataclasses.dataclass
class NodeGraph:
    """Node -> node neighbours and rigidity weights of an embedded graph, the
    arrays the ARAP regulariser reads (Skeletool/Mesh/EmbeddedGraph.cpp:
    155-167, 327-436, 460-490): per node an ascending neighbour list (the
    reference keeps them in a std::set) as a CSR, and the mean segmentation
    weight of the vertices connected to the node."""
    n2n_offsets: np.ndarray
    n2n_sizes: np.ndarray
    n2n_indices: np.ndarray
    rigidity: np.ndarray
    max_connections: int


def node_graph(verts: np.ndarray, graph: EmbeddedGraph, k: int, rng: np.random.Generator,
               refinement: bool = False, seg_weights: np.ndarray | None = None) -> NodeGraph:
    """Neighbours: the ``k`` nearest other nodes of every node, made
    symmetric (the reference takes the edges of its graph mesh, which are
    symmetric).  Rigidity: per-vertex segmentation weights (U[1, 40] unless
    given) averaged over each node's vertex connections, the ones below 20
    divided by 10 in the refinement mode (EmbeddedGraph.cpp:460-490)."""
    M = graph.n_nodes
    g = verts[graph.node_vertex].astype(np.float64)
    d = np.linalg.norm(g[:, None] - g[None], axis=2)
    np.fill_diagonal(d, np.inf)
    near = np.argsort(d, axis=1, kind="stable")[:, :k]
    nb = [set() for _ in range(M)]
    for j in range(M):
        for q in near[j]:
            nb[j].add(int(q))
            nb[int(q)].add(j)
    lists = [sorted(x) for x in nb]
    sizes = np.array([len(x) for x in lists], np.int32)
    offsets = np.zeros(M, np.int32)
    offsets[1:] = np.cumsum(sizes)[:-1]
    indices = np.array([q for x in lists for q in x], np.int32)
    if seg_weights is None:
        seg_weights = rng.uniform(1.0, 40.0, size=verts.shape[0]).astype(np.float32)
    rig = np.zeros(M, np.float32)
    cnt = np.zeros(M, np.float32)
    for v in range(verts.shape[0]):  # the reference's loop order: vertices, then their connections
        o, n = graph.v2n_offsets[v], graph.v2n_sizes[v]
        for e in graph.v2n_indices[o:o + n]:
            w = seg_weights[v]
            rig[e] = np.float32(rig[e] + (w / np.float32(10.0) if refinement and w < 20.0 else w))
            cnt[e] += 1
    rig = (rig / np.maximum(cnt, 1)).astype(np.float32)
    return NodeGraph(offsets, sizes, indices, rig, int(sizes.max()))


def eg_scene(subdiv: int, n_nodes: int, batch: int, seed: int, k: int = 4, n_markers: int = 8,
             delta_rot_std: float = 0.05, delta_t_std: float = 0.01 * MM, skinned_rot_std: float = 0.1,
             skinned_t_std: float = 0.02 * MM, disp_std: float = 0.001 * MM):
    """Embedded-graph inputs on a jittered icosphere: the graph (farthest-point
    nodes, K nearest nodes per vertex, inverse-distance weights), markers on
    random node vertices, and per-frame node rotations (Euler, rad) /
    translations (mm) and vertex displacements."""
    rng = rng_for(seed)
    verts, faces = sphere_mesh(subdiv, rng)
    g = embedded_graph(verts, n_nodes, k, rng)
    mk_nodes = rng.choice(n_nodes, size=n_markers, replace=False).astype(np.int32) if n_markers else None
    markers = (verts[g.node_vertex[mk_nodes]] + rng.normal(0, 5.0, (n_markers, 3))).astype(np.float32) \
        if n_markers else None
    f = lambda std, shape: rng.normal(0.0, std, size=shape).astype(np.float32)  # noqa: E731
    return dict(verts=verts, faces=faces, graph=g, markers=markers, marker_node=mk_nodes,
                dT=f(delta_t_std, (batch, n_nodes, 3)), dA=f(delta_rot_std, (batch, n_nodes, 3)),
                sT=f(skinned_t_std, (batch, n_nodes, 3)), sA=f(skinned_rot_std, (batch, n_nodes, 3)),
                disp=f(disp_std, (batch, verts.shape[0], 3)))


def skinning_scene(subdiv: int, n_skel: int, batch: int, seed: int, k: int = 4, pose_amplitude: float = 0.5):
    """Skinned-character inputs: jittered icosphere, random revolute tree
    (three joints per skeletal joint), K nearest skinning joints per vertex
    with Dirichlet weights, per-frame poses U(-a, a) and small displacements."""
    rng = rng_for(seed)
    verts, faces = sphere_mesh(subdiv, rng)
    sk = random_skeleton(n_skel, rng)
    idx, w = skinning_weights(verts, sk, k, rng)
    dofs = np.stack([random_pose(sk, rng_for(seed, b), pose_amplitude) for b in range(batch)])
    return dict(verts=verts, faces=faces, skeleton=sk, skin_index=idx, weights=np.tile(w[None], (batch, 1, 1)),
                dofs=dofs, disp=rng.normal(0.0, 1.0, size=(batch, verts.shape[0], 3)).astype(np.float32))


def ellipse_dt(width: int, height: int, r: np.random.Generator, scale: float = 1.0) -> np.ndarray:
    """uint8 distance-transform image [H,W] of a random ellipse (centre +-64 px,
    semi-axes U[80,200] px at 512 px, scaled by ``scale``)."""
    cx = width / 2 + r.uniform(-64, 64) * scale
    cy = height / 2 + r.uniform(-64, 64) * scale
    a, bb = r.uniform(80, 200) * scale, r.uniform(80, 200) * scale
    th = r.uniform(0, np.pi)
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    x, y = xx + 0.5 - cx, yy + 0.5 - cy
    u = (math.cos(th) * x + math.sin(th) * y) / a
    v = (-math.sin(th) * x + math.cos(th) * y) / bb
    return encode_dt((u * u + v * v) <= 1.0)


def silhouette_masks(batch: int, views: int, width: int, height: int, seed: int, scale: float = 1.0) -> np.ndarray:
    """uint8 distance-transform images [B,C,H,W] of seeded random ellipses
    (centre +-64 px, semi-axes U[80,200] px at 512 px, scaled by ``scale``)."""
    out = np.empty((batch, views, height, width), np.uint8)
    for b in range(batch):
        for c in range(views):
            out[b, c] = ellipse_dt(width, height, rng_for(seed, 100 * b + c), scale)
    return out


# per-view image sizes of the batched mixed-resolution configuration (W x H)
MIXED_SIZES = ((512, 512), (768, 1024), (1024, 1024), (1536, 1024))


def mixed_camera_sizes(views: int, seed: int) -> tuple[list[int], list[int]]:
    """Per-camera (widths, heights) drawn uniformly from MIXED_SIZES."""
    r = rng_for(seed, 999)
    pick = r.integers(0, len(MIXED_SIZES), size=views)
    return [MIXED_SIZES[k][0] for k in pick], [MIXED_SIZES[k][1] for k in pick]


def identity_crops(batch: int, views: int, width: int, height: int) -> np.ndarray:
    """Multi-view crops (border u, border v, scale, min u, min v, max u, max v) of uncropped images."""
    c = np.array([0, 0, 1, 0, 0, width, height], np.float32)
    return np.tile(c, (batch, views, 1))


def chain_scene(subdiv: int, n_nodes: int, n_skel: int, frames: int, views: int, width, height, seed: int,
                fx: float | None = None, ring_radius: float = 3.0 * MM, k: int = 4, pose_amplitude: float = 0.5,
                delta_rot_std: float = 0.05, delta_t_std: float = 0.01 * MM, n_masks: int | None = None,
                first_frame: int = 0) -> dict:
    """Inputs of the whole deform-and-render chain on one character: a
    jittered icosphere with an embedded graph (``n_nodes`` farthest-point
    nodes, K nearest nodes per vertex) and a random ``n_skel``-joint tree with
    K-nearest-joint skinning weights; per frame an independent pose (joint
    angles U(-a, a)) and node deltas (Euler N(0, 0.05) rad, translation
    N(0, 10) mm); 8 markers on random nodes; cameras on a ring; vertex colours U[0,1] (one set for
    all frames: the character's appearance); 8-bit target
    images (``target_u8`` uniform bytes, ``target`` = byte / 255 in float32, the value
    ``hc_image_u8_to_f32`` computes on the device); silhouette distance-transform images of
    seeded random ellipses (``n_masks`` distinct ones, default one per view, reused across frames).

    ``width`` / ``height`` may be per-camera sequences: each camera then has
    its own image size, focal length fx = fy = 600 min(W, H) / 512 (unless
    ``fx`` is given) and centred principal point, and the per-pixel arrays
    (``target``, ``target_u8``, ``dt``) are [B, pixels of a frame, ...] with
    the frame's cameras concatenated in order.

    ``frames`` frames starting at frame ``first_frame`` of the seed's
    sequence: the character, cameras and masks depend on the seed alone and
    every per-frame input on (seed, frame), so ``chain_scene(..., frames=n,
    first_frame=f)`` equals frames f .. f+n-1 of a longer scene."""
    rng = rng_for(seed)
    verts, faces = sphere_mesh(subdiv, rng)
    N = verts.shape[0]
    graph = embedded_graph(verts, n_nodes, k, rng)
    mk_nodes = rng.choice(n_nodes, size=8, replace=False).astype(np.int32)
    markers = (verts[graph.node_vertex[mk_nodes]] + rng.normal(0, 5.0, (8, 3))).astype(np.float32)
    sk = random_skeleton(n_skel, rng)
    skin_idx, skin_w = skinning_weights(verts, sk, k, rng)
    fr = range(first_frame, first_frame + frames)
    dofs = np.stack([random_pose(sk, rng_for(seed, b), pose_amplitude) for b in fr])
    sized = np.ndim(width) > 0 or np.ndim(height) > 0
    ws = [int(x) for x in np.broadcast_to(np.asarray(width), (views,))]
    hs = [int(x) for x in np.broadcast_to(np.asarray(height), (views,))]
    nm = views if n_masks is None else n_masks
    if not sized:
        W, H = ws[0], hs[0]
        if fx is None:
            fx = 600.0 * min(W, H) / 512.0
        ex, it = camera_ring(views, ring_radius, fx, W, H)
        masks = silhouette_masks(1, nm, W, H, seed=seed, scale=min(W, H) / 512.0)[0]
        dt = np.stack([masks[np.arange(views) % nm]] * frames)
        crops = identity_crops(frames, views, W, H)
    else:
        ex, it = [], []
        for c in range(views):
            f_c = fx if fx is not None else 600.0 * min(ws[c], hs[c]) / 512.0
            e1, i1 = camera_ring(views, ring_radius, f_c, ws[c], hs[c])
            ex.append(e1[12 * c:12 * c + 12])
            it.append(i1[9 * c:9 * c + 9])
        ex, it = np.concatenate(ex), np.concatenate(it)
        masks = [ellipse_dt(ws[c], hs[c], rng_for(seed, c % nm), min(ws[c], hs[c]) / 512.0).reshape(-1)
                 for c in range(views)]
        dt = np.stack([np.concatenate(masks)] * frames)
        crops = np.stack([np.stack([np.array([0, 0, 1, 0, 0, ws[c], hs[c]], np.float32) for c in range(views)])]
                         * frames)
    P_frame = int(sum(w * h for w, h in zip(ws, hs)))
    # the appearance is shared by all frames (one parameter, its gradient
    # summed over frames and ranks); pose, node deltas, lighting and targets
    # are per frame
    colors = rng.uniform(0.0, 1.0, size=(N, 3)).astype(np.float32)
    texture = rng.uniform(0.0, 1.0, size=(16, 16, 3)).astype(np.float32)
    per = {key: [] for key in ("dT", "dA", "sh", "target_u8")}
    for b in fr:
        r = frame_rng(seed, b)
        per["dT"].append(r.normal(0.0, delta_t_std, size=(n_nodes, 3)).astype(np.float32))
        per["dA"].append(r.normal(0.0, delta_rot_std, size=(n_nodes, 3)).astype(np.float32))
        per["sh"].append(sh_coefficients(views, r))
        shape = (P_frame, 3) if sized else (views, hs[0], ws[0], 3)
        per["target_u8"].append(r.integers(0, 256, size=shape, dtype=np.uint8))
    per = {key: np.stack(v) for key, v in per.items()}
    target_u8 = per["target_u8"]
    return dict(verts=verts, faces=faces, graph=graph, markers=markers, marker_node=mk_nodes, skeleton=sk,
                skin_index=skin_idx, skin_weights=skin_w,
                dofs=dofs, dT=per["dT"], dA=per["dA"],
                disp=np.zeros((frames, N, 3), np.float32),
                colors=np.tile(colors[None], (frames, 1, 1)), texture=np.tile(texture[None], (frames, 1, 1, 1)),
                sh=per["sh"],
                extr=np.tile(ex[None], (frames, 1)), intr=np.tile(it[None], (frames, 1)),
                texcoords=spherical_uvs(verts, faces),
                target=target_u8.astype(np.float32) / np.float32(255.0), target_u8=target_u8,
                dt=dt, crops=crops,
                N=N, F=faces.shape[0], M=n_nodes, B=frames, C=views, W=ws if sized else ws[0],
                H=hs if sized else hs[0], P_frame=P_frame, first_frame=first_frame)
