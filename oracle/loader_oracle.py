"""Test infrastructure: a literal, loop-by-loop restatement of the reference's
embedded-graph construction, used only to check the vectorised loader in
``deepcharacters_b200.loaders`` on small meshes.

Follows CustomTensorFlowCPPOperators/src/Skeletool/Mesh/EmbeddedGraph.cpp:
setupNodeGraph :33-180, computeConnections :182-302, normalizeWeights
:304-321, initializeGPUMemory :379-548 (table layout, rigidity, markers), with
trimesh.cpp:868-911 (breadth-first hop distance over the face neighbours).

Parity unpinned: the reference ships no character or graph files and its
loaders need Eigen, which is absent, so neither can be run here.  This
restatement is checked against hand-worked cases in the tests.
"""
from __future__ import annotations

import collections
import math

import numpy as np

UNREACHED = 1000000


def neighbours(n, faces):
    nb = [set() for _ in range(n)]
    for a, b, c in faces:
        a, b, c = int(a), int(b), int(c)
        nb[a].update((b, c))
        nb[b].update((a, c))
        nb[c].update((a, b))
    return nb


def hops(nb, src):
    d = [UNREACHED] * len(nb)
    d[src] = 0
    q = collections.deque([src])
    while q:
        v = q.popleft()
        for u in sorted(nb[v]):
            if d[u] == UNREACHED:
                d[u] = d[v] + 1
                q.append(u)
    return d


def f32(x):
    return float(np.float32(x))


def norm3(a, b):
    d = [np.float32(a[i]) - np.float32(b[i]) for i in range(3)]
    return f32(np.sqrt(np.float32(np.float32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])))


def extreme_y(v):
    hi = lo = -1
    maxy, miny = f32(-10000.0), f32(100000.0)
    for i in range(len(v)):
        if v[i][1] > maxy:
            maxy, hi = v[i][1], i
        if v[i][1] < miny:
            miny, lo = v[i][1], i
    return hi, lo


def build_graph(verts, faces, gverts, gfaces, seg_weights, markers, refinement=False):
    """Returns a dict of the reference's host tables for the graph."""
    V = [tuple(float(x) for x in p) for p in np.asarray(verts, np.float32)]
    G = [tuple(float(x) for x in p) for p in np.asarray(gverts, np.float32)]
    N, M = len(V), len(G)
    nb = neighbours(N, faces)
    gnb = neighbours(M, gfaces)
    hi, lo = extreme_y(V)
    dhi, dlo = hops(nb, hi), hops(nb, lo)
    ghi, glo = extreme_y(G)
    gdhi, gdlo = hops(gnb, ghi), hops(gnb, glo)
    used = [False] * N
    node = []
    for vl in range(M):
        best, bid = f32(np.finfo(np.float32).max), -1
        for vh in range(N):
            dist = norm3(G[vl], V[vh])
            same = ((gdhi[vl] != UNREACHED) == (dhi[vh] != UNREACHED)) and \
                   ((gdlo[vl] != UNREACHED) == (dlo[vh] != UNREACHED))
            if dist < best and not used[vh] and same:
                best, bid = dist, vh
        used[bid] = True
        node.append(bid)
    emb_nb = [sorted(gnb[n]) for n in range(M)]
    dist = [hops(nb, node[n]) for n in range(M)]
    radius = []
    for n in range(M):
        r = 0
        for j in emb_nb[n]:
            r = max(r, dist[n][node[j]])
        r //= 2
        radius.append(max(r, 3))
    conn = []
    for v in range(N):
        c = []
        for i in range(M):
            d = f32(np.float32(dist[i][v]) / np.float32(radius[i]))
            if d <= 1:
                c.append([i, f32(math.exp(-0.5 * d * d))])
        if not c:
            dmin, imin = f32(1000000.0), -1
            for i in range(M):
                d = f32(dist[i][v])
                if d <= dmin:
                    dmin, imin = d, i
            c.append([imin, 1.0])
        conn.append(c)
    for c in conn:
        w = np.float32(0.0)
        for _, x in c:
            w = np.float32(w + np.float32(x))
        for e in c:
            e[1] = f32(np.float32(e[1]) / w)
    n2v = [[(v, w) for v in range(N) for (i, w) in conn[v] if i == k] for k in range(M)]
    rig = []
    for k in range(M):
        s, cnt = np.float32(0.0), np.float32(0.0)
        for v in range(N):
            for i, _ in conn[v]:
                if i == k:
                    w = np.float32(seg_weights[v])
                    s = np.float32(s + (w / np.float32(10.0) if refinement and w < 20.0 else w))
                    cnt = np.float32(cnt + 1)
        rig.append(f32(s / cnt))
    marker_node = []
    for m in np.asarray(markers, np.float32).reshape(-1, 3):
        best, bid = f32(np.finfo(np.float32).max), -1
        for n in range(M):
            d = norm3(m, V[node[n]])
            if d < best:
                best, bid = d, n
        marker_node.append(bid)
    return dict(node_vertex=node, radius=radius, conn=conn, n2v=n2v, n2n=emb_nb, rigidity=rig,
                marker_node=marker_node)
