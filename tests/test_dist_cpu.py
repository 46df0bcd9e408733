"""Data-parallel host logic on CPU: two gloo ranks (world size 2).

The frames of a step are sharded over the ranks; the shared vertex-colour
gradient summed over the ranks must equal the single-process gradient over
all frames.  The per-frame gradient here is the FP64 oracle's adjoint of the
vertex-colour interpolation (a sum over pixels of G * barycentric weight per
vertex), computed on synthetic face / barycentric buffers."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from deepcharacters_b200 import dist as D


def colour_grad(face, bary, G, faces, n_vertices):
    """d loss / d vertex colours for vertexColor shadeless: sum over covered
    pixels of G times the pixel's barycentric weight, per vertex."""
    out = np.zeros((n_vertices, 3))
    m = face >= 0
    f = faces[face[m]]
    w = np.stack([bary[m][:, 0], bary[m][:, 1], 1.0 - bary[m][:, 0] - bary[m][:, 1]], 1)
    for k in range(3):
        np.add.at(out, f[:, k], G[m] * w[:, k:k + 1])
    return out


def frame_data(frame, n_vertices=50, n_faces=80, H=12, W=10):
    rng = np.random.default_rng(1000 + frame)
    faces = np.random.default_rng(7).integers(0, n_vertices, size=(n_faces, 3))
    face = rng.integers(-1, n_faces, size=(H, W))
    bary = rng.uniform(0, 0.5, size=(H, W, 2))
    G = rng.normal(size=(H, W, 3))
    return face, bary, G, faces


def _worker(rank, world, port, total, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    try:
        w, r, _ = D.init("gloo", timeout_s=60)
        first, count = D.shard_frames(total, w, r)
        g = np.zeros((50, 3))
        for fr in range(first, first + count):
            g += colour_grad(*frame_data(fr), 50)
        t = torch.from_numpy(g)
        D.allreduce_shared([t], w)
        mx = D.max_over_ranks(float(r + 1), w)
        D.barrier(w)
        q.put((r, first, count, t.numpy(), mx))
        D.finalize(w)
    except Exception as e:  # report, do not hang the parent
        q.put((rank, "error", repr(e), None, None))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_frames_covers_every_frame_once():
    for total in (1, 5, 16, 17):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                first, count = D.shard_frames(total, world, r)
                seen += list(range(first, first + count))
            assert seen == list(range(total)), (total, world)


@pytest.mark.timeout(120)
def test_two_gloo_ranks_sum_to_the_single_process_gradient():
    total, world = 5, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, total, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=100) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
    res.sort(key=lambda x: x[0])
    assert all(x[1] != "error" for x in res), res
    ref = sum(colour_grad(*frame_data(fr), 50) for fr in range(total))
    for r, first, count, g, mx in res:
        assert np.allclose(g, ref, rtol=1e-12, atol=1e-12)
        assert mx == float(world)
    assert [x[2] for x in res] == [3, 2]
