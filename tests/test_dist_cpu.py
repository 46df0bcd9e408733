"""Data-parallel host logic on CPU: two gloo ranks (world size 2), driving
the code path ``bench.py`` uses on GPUs.

Each rank takes its block of frames (``dist.shard_frames``), generates only
those frames of the scene (``synthetic.chain_scene(first_frame=...)``),
builds the product's ``DeformRenderChain`` on them (library calls recorded,
not run: there is no GPU here), fills the chain's per-frame vertex-colour
gradient buffer with the FP64 oracle's adjoint of those frames (node
skinning -> EG -> raster -> L1 -> raster adjoint) and reduces it with
``dist.shared_gradient``, the call the benchmark makes after every step.  The
result on every rank must equal the single-process gradient over all frames.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from deepcharacters_b200 import dist as D
from deepcharacters_b200 import synthetic as S

SCENE = dict(subdiv=2, n_nodes=20, n_skel=4, views=2, width=48, height=48, seed=3)


def scene(frames, first_frame=0):
    p = SCENE
    return S.chain_scene(p["subdiv"], p["n_nodes"], p["n_skel"], frames, p["views"], p["width"], p["height"],
                         seed=p["seed"], first_frame=first_frame)


def oracle_colour_grads(sc):
    """[B,N,3] d L1 / d vertex colours per frame, FP64 oracle end to end."""
    from deepcharacters_b200.chain import character, eg_data
    from oracle import oracle as O
    from oracle import skinning_oracle as K
    B, C, W, H = sc["B"], sc["C"], sc["W"], sc["H"]
    sT, sA, _ = K.pose2eg(character(sc), sc["dofs"], sc["graph"].node_vertex, sc["skin_weights"])
    v = O.eg_forward(eg_data(sc), sc["dT"], sc["dA"], sT.astype(np.float32), sA.astype(np.float32), sc["disp"],
                     precision="f64")["vertices"]
    fw = O.render_forward(sc["faces"], sc["texcoords"], B, C, W, H, "vertexColor", "shadeless", v, sc["colors"],
                          sc["texture"], sc["sh"], sc["extr"], sc["intr"], precision="f64", fragile=False)
    out = np.zeros((B, sc["N"], 3), np.float32)
    for b in range(B):  # the L1 is normalised per frame's call here; any per-frame gradient image serves
        d = 255.0 * (fw["render"][b:b + 1] - sc["target"][b:b + 1]) * (fw["face"][b:b + 1] >= 0)[..., None]
        g = (255.0 * np.sign(d) / max(int(np.count_nonzero(d)), 1)).astype(np.float32)
        bw = O.render_backward(sc["faces"], sc["texcoords"], 1, C, W, H, "vertexColor", "shadeless", g, v[b:b + 1],
                               sc["colors"][b:b + 1], sc["texture"][b:b + 1], sc["sh"][b:b + 1],
                               sc["target"][b:b + 1], fw["vnormal"][b:b + 1], fw["bary"][b:b + 1],
                               fw["face"][b:b + 1], sc["extr"][b:b + 1], sc["intr"][b:b + 1], precision="f64")
        out[b] = bw["vertex_color_grad"][0]
    return out


def _worker(rank, world, port, total, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    try:
        from deepcharacters_b200 import _lib
        import deepcharacters_b200.chain as chain
        _lib.call = lambda *a: None  # no GPU: the chain's library calls are not run
        chain._stream = lambda: 0
        w, r, _ = D.init("gloo", timeout_s=60)
        first, count = D.shard_frames(total, w, r)
        sc = scene(count, first)
        ch = chain.DeformRenderChain(sc, "cpu", count, sc["C"], sc["W"], sc["H"])
        ch.buf["gcol"].copy_(torch.from_numpy(oracle_colour_grads(sc)))
        out = torch.empty(ch.buf["gcol"].shape[1:])
        D.shared_gradient(ch.buf["gcol"], out, w)
        mx = D.max_over_ranks(float(r + 1), w)
        D.barrier(w)
        q.put((r, first, count, out.numpy(), mx))
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
    # weak scaling: every rank gets the same number of frames
    assert [D.rank_frames(16, 8, r) for r in range(8)] == [(16 * r, 16) for r in range(8)]


def test_rank_scene_is_the_slice_of_the_whole_job():
    whole = scene(5)
    for first, count in ((0, 2), (2, 3), (4, 1)):
        part = scene(count, first)
        for k in ("dofs", "dT", "dA", "colors", "texture", "sh", "target_u8", "dt", "extr", "intr", "crops"):
            assert np.array_equal(part[k], whole[k][first:first + count]), k
        assert np.array_equal(part["verts"], whole["verts"]) and np.array_equal(part["faces"], whole["faces"])


@pytest.mark.timeout(180)
def test_two_gloo_ranks_sum_to_the_single_process_gradient():
    total, world = 3, 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, total, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=160) for _ in range(world)]
    for p in procs:
        p.join(timeout=30)
    res.sort(key=lambda x: x[0])
    assert all(x[1] != "error" for x in res), res
    ref = oracle_colour_grads(scene(total)).astype(np.float64).sum(0)
    assert np.abs(ref).max() > 0
    for r, first, count, g, mx in res:
        assert np.allclose(g, ref, rtol=1e-5, atol=1e-6 * np.abs(ref).max()), np.abs(g - ref).max()
        assert mx == float(world)
    assert [(x[1], x[2]) for x in res] == [(0, 2), (2, 1)]
