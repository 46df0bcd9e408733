#!/usr/bin/env python
"""Benchmark of the deform-and-render chain: fwd+bwd views/s at 81,920 triangles, 1024x1024.

Workload (one "step"): the deform-and-render chain on 16 frames x 8 views of
a character built on an icosphere subdivision-6 mesh (40,962 vertices /
81,920 triangles, radius 1 m = 1000 units, 1 cm vertex jitter): node skinning
of a 1000-node embedded graph by a 24-joint tree (3 revolute dofs each),
embedded-graph deformation, vertex-colour rasterization at 1024x1024 from
cameras on a 3 m ring (fx = fy = 1200), the masked L1 image loss, camera
projection + projected-mesh boundary + the silhouette distance-transform loss,
and the adjoints back to node rotations / translations and vertex colours.
Synthetic data; inputs larger than L2 (1.6 GB of target images per step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:       the chain through libhc.so, captured once in a CUDA graph and
            replayed (value: device time, inputs resident in HBM); e2e runs the
            same step through the public Python API with every step's inputs
            copied from pinned host memory and the loss read back.
reference:  the reference's own CUDA kernels (compiled unmodified for sm_100a
            into oracle/_ref) driven op by op like its TF ops (the renderer
            per frame), node skinning on the host as the reference's CPU op,
            the losses as elementwise torch ops: the plain per-op path.
Under torchrun every rank runs its own 16 frames (weak scaling); the
gradient of the shared vertex colours is all-reduced over NCCL each step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

from deepcharacters_b200 import dist as D  # noqa: E402

METRIC = "fwd+bwd views/s at 81,920 tris 1024²: batched/graph vs plain per-view (same B200)"
FRAMES, VIEWS, RES, SUBDIV = 16, 8, 1024, 6


def algorithmic_bytes_per_view(N, F, H, W, V):
    """Compulsory HBM traffic per view of the fused fwd+bwd chain:
    target RGB 12 + distance image 1 + tri-id 4 + barycentrics 8 written,
    tri-id / barycentrics 12 read back = 37 B per pixel, plus per-frame mesh
    data (positions / colours fwd+bwd, faces, skinning tables, gradients)
    amortised over the V views of a frame."""
    return 37 * H * W + (136 * N + 24 * F) / V


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm = [float(r[0]) for r in self.rows if len(r) >= 8 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 8 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 8:
                continue
            for i, n in enumerate(names):
                if r[4 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# distributed plumbing
# --------------------------------------------------------------------------
def dist_setup(gpus: int):
    world, rank, local = D.env_rank()
    torch.cuda.set_device(local if world > 1 else 0)
    return D.init("nccl", timeout_s=120, device=torch.device("cuda", local))


def barrier(world):
    D.barrier(world)


def max_over_ranks(x: float, world: int) -> float:
    return D.max_over_ranks(x, world, "cuda")


# --------------------------------------------------------------------------
# workload
# --------------------------------------------------------------------------
N_NODES, N_SKEL, FX = 1000, 24, 1200.0
W_SIL, W_SIL1 = 1e-3, 1e-3  # weights of the two silhouette residual terms


def make_workload(rank: int):
    from deepcharacters_b200 import synthetic as S
    return S.chain_scene(SUBDIV, N_NODES, N_SKEL, FRAMES, VIEWS, RES, RES, seed=2 + 100 * rank, fx=FX)


def cpu_baseline(sc, frames=1, views=2):
    """The oracle restatement on the host cores (bounded sample): node
    skinning + EG forward, raster + L1 + raster adjoint + EG adjoint in float."""
    from deepcharacters_b200.chain import character, eg_data
    from oracle import oracle as O
    from oracle import skinning_oracle as K
    B, C = frames, views
    d = eg_data(sc)
    ch = character(sc)
    cores = os.cpu_count() or 1
    extr = sc["extr"][:B, :12 * C]
    intr = sc["intr"][:B, :9 * C]
    t0 = time.perf_counter()
    sT, sA, _ = K.pose2eg(ch, sc["dofs"][:B], sc["graph"].node_vertex, sc["skin_weights"])
    eg = O.eg_forward(d, sc["dT"][:B], sc["dA"][:B], sT.astype(np.float32), sA.astype(np.float32), sc["disp"][:B],
                      precision="f32")
    verts = eg["vertices"]
    fw = O.render_forward(sc["faces"], sc["texcoords"], B, C, RES, RES, "vertexColor", "shadeless", verts,
                          sc["colors"][:B], sc["texture"][:B], sc["sh"][:B, :C], extr, intr, precision="f32",
                          nthreads=cores, fragile=False)
    m = (fw["face"] >= 0)[..., None]
    diff = 255.0 * (fw["render"] - sc["target"][:B, :C]) * m
    cnt = max(int(np.count_nonzero(diff)), 1)
    g = (255.0 * np.sign(diff) / cnt).astype(np.float32)
    bw = O.render_backward(sc["faces"], sc["texcoords"], B, C, RES, RES, "vertexColor", "shadeless", g, verts,
                           sc["colors"][:B], sc["texture"][:B], sc["sh"][:B, :C], sc["target"][:B, :C], fw["vnormal"],
                           fw["bary"], fw["face"], extr, intr, precision="f32", nthreads=cores)
    O.eg_backward(d, bw["vertex_pos_grad"], np.zeros((B, 8, 3), np.float32), sc["dT"][:B], sc["dA"][:B],
                  sA.astype(np.float32), sc["disp"][:B], precision="f32")
    dt = time.perf_counter() - t0
    return {"value": B * C / dt, "unit": "views/s", "cores": cores, "kind": "port",
            "sample": f"{B} frame x {C} views of the same workload: node skinning + EG fwd, raster + L1 + raster "
                      "adjoint + EG adjoint (float oracle, OpenMP; silhouette terms not in the sample)"}


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def stage_bytes(sc):
    """Algorithmic bytes per call of each stage (compulsory traffic of what
    the stage must read and write once)."""
    B, C, P, N, F, M = FRAMES, VIEWS, RES * RES, sc["N"], sc["F"], sc["M"]
    K = 4
    eg = B * (12 * N * 2 + 8 * K * N + 24 * M) + 12 * N  # read base / write verts + normals, CSR, node params
    return {
        # EG + raster: verts read, bary 8 + face 4 + render 12 written per pixel; the fused L1 reads the
        # target (counted for every pixel here)
        "deform_render_forward": eg + B * C * (24 * P + 12 * N) + B * C * 12 * P,
        # projection, coverage + boundary, per-pixel silhouette residual (dt 1, res1 8, closest 4), squared loss
        "silhouette_forward": B * C * (16 * N + 1 * P + 1 * P + 12 * P + 8 * P + 8 * 3 * N),
        "silhouette_backward": B * C * (8 * P + 4 * P + 24 * N) + B * 24 * N,
        # bwd raster reads render 12 (the fused L1 gradient) + bary 8 + face 4 + target 12 per pixel,
        # writes vertex grads; EG adjoint
        "render_eg_backward": B * C * 36 * P + B * (36 * N + 24 * N) + eg,
    }


def kernel_bytes(sc, covered):
    """Algorithmic bytes per launch of the two raster kernels over FRAMES x VIEWS views
    with the image L1 fused in (``covered`` = pixels with a face, all views):
    k_resolve writes face 4 + barycentrics 8 + colour 12 B per pixel, reads the
    target (12 B) of the covered pixels and each frame's positions, colours and
    faces once; k_render_grad reads the render 12 (the image gradient is formed
    from it), barycentrics 8, face 4 and target 12 B per pixel and each frame's
    positions, colours and faces, and writes the position and colour gradients."""
    V, P, N, F = FRAMES * VIEWS, RES * RES, sc["N"], sc["F"]
    return {"resolve": V * 24 * P + 12 * covered + FRAMES * (24 * N + 12 * F),
            "render_grad": V * 36 * P + FRAMES * (24 * N + 12 * F + 24 * N)}


def run_ours(args, world, rank, local):
    from deepcharacters_b200 import _lib
    dev = torch.device("cuda", local)
    from deepcharacters_b200.chain import DeformRenderChain
    sc = make_workload(rank)
    ch = DeformRenderChain(sc, dev, FRAMES, VIEWS, RES, RES, W_SIL, W_SIL1)
    views_per_step = FRAMES * VIEWS
    # autotuner: raster tile size and bin capacity (untimed)
    tune = ch.autotune() if not args.no_autotune else {}
    binned, spilled = ch.check()  # raises if the raster's spill capacity overflowed
    # eager warm-up (allocates every workspace), then capture one step
    for _ in range(2):
        ch.step()
    torch.cuda.synchronize()
    l0 = _lib.lib().hc_kernel_launches()
    g = ch.capture_step()
    launches_per_step = _lib.lib().hc_kernel_launches() - l0
    torch.cuda.synchronize()

    def allreduce():  # the shared vertex-colour gradient; frames are sharded
        D.allreduce_shared([ch.buf["gcol"]], world)

    for _ in range(args.warmup):
        g.replay()
        allreduce()
    torch.cuda.synchronize()
    barrier(world)
    clk = ClockSampler(local)
    clk.start()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    st.record()
    for _ in range(args.steps):
        g.replay()
        allreduce()
    en.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(st.elapsed_time(en) / args.steps, world)
    barrier(world)
    value = views_per_step * world / (ms / 1e3)

    # per-stage device time (eager, same inputs) for the roofline of the dominant call
    stage_ms = {}
    for name, fn in ch.stages():
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(3):
            fn()
        b.record()
        torch.cuda.synchronize()
        stage_ms[name] = a.elapsed_time(b) / 3
    sbytes = stage_bytes(sc)
    N, F = sc["N"], sc["F"]
    # per-kernel device time of the two raster kernels (events around each launch, eager)
    ch.rend.set_kernel_timing(True)
    kern_ms = {}
    for _ in range(3):
        ch.forward()
        ch.backward()
        kt = ch.rend.kernel_times()
        for k in ("resolve", "render_grad"):
            kern_ms.setdefault(k, []).append(kt[k])
    ch.rend.set_kernel_timing(False)
    kern_ms = {k: sum(v) / len(v) for k, v in kern_ms.items()}
    kbytes = kernel_bytes(sc, int((ch.buf["face"] >= 0).sum()))
    dom = max(kern_ms, key=kern_ms.get)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    ach = kbytes[dom] / (kern_ms[dom] / 1e3) / 1e9
    traffic_path = os.path.join(ROOT, "profiles", "traffic.json")
    traffic = None
    if os.path.exists(traffic_path):
        tj = json.load(open(traffic_path)).get("k_" + dom)
        if tj:  # ncu DRAM bytes per view of a smaller capture, scaled to this launch's views
            traffic = tj["dram_bytes_per_view"] * FRAMES * VIEWS

    # e2e: public API, pinned host inputs copied every step, losses read back
    e2e = None if args.no_e2e else run_e2e(ch, sc, dev, args, world)

    line = {
        "metric": METRIC, "value": value, "unit": "views/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded icosphere character, random pose / node deltas, ring cameras, random targets, "
                "ellipse silhouettes)",
        "config": {"workload": "deform-and-render chain fwd+bwd: icosphere subdiv-6 (40,962 verts / 81,920 tris), "
                               "1000-node embedded graph (K=4) skinned by a 24-joint tree (node DQ), 16 frames x 8 "
                               "views 1024x1024, vertexColor raster + masked L1 + silhouette DT loss, gradients to "
                               "node rotations / translations and vertex colours, one CUDA graph per step",
                   "frames": FRAMES, "views": VIEWS, "resolution": [RES, RES], "triangles": F, "vertices": N,
                   "nodes": N_NODES, "joints": 3 * N_SKEL,
                   "parallelism": f"frames sharded, {world} rank(s)",
                   "l2": "inputs larger than L2 (1.6 GB of target images per step)",
                   "raster_tile": ch.tuning[0], "bin_capacity": ch.tuning[1],
                   "autotune_ms": {f"{t}x{c}": round(v, 3) for (t, c), v in tune.items()},
                   "bin_pairs": binned, "spilled_pairs": spilled},
        "e2e": e2e,
        "gpu_launches": int(launches_per_step * args.steps),
        "roofline": {"bound": "hbm", "kernel": "k_" + dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650",
                     "kernel_ms": kern_ms, "kernel_bytes": kbytes,
                     "stage_ms": stage_ms, "stage_bytes": sbytes,
                     "chain_bytes_per_view": algorithmic_bytes_per_view(N, F, RES, RES, VIEWS),
                     "chain_frac": algorithmic_bytes_per_view(N, F, RES, RES, VIEWS) * value / world / 1e9 / peak},
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sc)
    if rank == 0:
        print(json.dumps(line), flush=True)


E2E_KEYS = ("dofs", "dT", "dA", "colors", "sh", "extr", "intr", "target_u8", "dt")


def run_e2e(ch, sc, dev, args, world):
    """Same step through the C ABI with host inputs: per step H2D of the pose,
    node deltas, vertex colours, cameras, SH, the 8-bit target images
    (widened to float32 on the device by ``hc_image_u8_to_f32``, the same
    values as the resident float targets) and distance images from pinned
    memory (double-buffered on a copy stream), and D2H of the three loss
    values."""
    from deepcharacters_b200 import _lib
    host = {k: torch.from_numpy(np.ascontiguousarray(sc[k])).pin_memory() for k in E2E_KEYS}
    bufs = []
    for _ in range(2):
        b = {k: torch.empty_like(ch.inp[k]) for k in E2E_KEYS if k != "target_u8"}
        b["target_u8"] = torch.empty(host["target_u8"].shape, dtype=torch.uint8, device=dev)
        b["target"] = torch.empty_like(ch.inp["target"])
        bufs.append(b)
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    copy = torch.cuda.Stream()
    loss_host = torch.zeros((3,), dtype=torch.float32).pin_memory()
    ready = [torch.cuda.Event() for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]
    saved = dict(ch.inp)

    def upload(slot):
        with torch.cuda.stream(copy):
            copy.wait_event(done[slot])
            for k in E2E_KEYS:
                bufs[slot][k].copy_(host[k], non_blocking=True)
            t8 = bufs[slot]["target_u8"]
            _lib.call("hc_image_u8_to_f32", copy.cuda_stream, t8.numel(), t8.data_ptr(),
                      bufs[slot]["target"].data_ptr())
            ready[slot].record(copy)

    # one captured step per input slot (the graphs read that slot's buffers)
    graphs = [ch.capture_step({k: v for k, v in bufs[slot].items() if k != "target_u8"}) for slot in range(2)]
    torch.cuda.synchronize()

    def run(n):
        for i in range(2):
            done[i].record()
        upload(0)
        for i in range(n):
            slot = i % 2
            torch.cuda.current_stream().wait_event(ready[slot])
            if i + 1 < n:
                upload((i + 1) % 2)
            graphs[slot].replay()
            D.allreduce_shared([ch.buf["gcol"]], world)
            done[slot].record()
            loss_host.copy_(ch.loss, non_blocking=True)
        torch.cuda.synchronize()

    run(max(args.warmup, 1))
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run(args.steps)
    dt = max_over_ranks(time.perf_counter() - t0, world)
    ch.inp.update(saved)
    return {"value": FRAMES * VIEWS * world * args.steps / dt, "unit": "views/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": 12, "ms_per_step": dt / args.steps * 1e3,
            "path": "DeformRenderChain.capture_step graphs (one per input slot) replayed per step, inputs copied "
                    "from pinned host memory on a copy stream (double buffer), target images as 8-bit RGB widened "
                    "on the device, losses read back"}


# --------------------------------------------------------------------------
# reference arm
# --------------------------------------------------------------------------
def run_reference(args, world, rank, local):
    if rank != 0:
        return
    from oracle import oracle as O
    if not (O.ref_available() and os.path.exists(O.REF_MB_LIB)):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref reference kernels were not built"}))
        return
    from oracle.chain_ref import RefChain
    dev = torch.device("cuda", local)
    sc = make_workload(0)
    ref = RefChain(sc, dev, FRAMES, VIEWS, RES, RES, W_SIL, W_SIL1)

    def step():
        ref.step()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    clocks = clk.stop()
    value = FRAMES * VIEWS * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "views/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "deform-and-render chain fwd+bwd: icosphere subdiv-6 (40,962 verts / 81,920 tris), "
                               "1000-node embedded graph (K=4) skinned by a 24-joint tree (node DQ), 16 frames x 8 "
                               "views 1024x1024, vertexColor raster + masked L1 + silhouette DT loss, gradients to "
                               "node rotations / translations and vertex colours",
                   "frames": FRAMES, "views": VIEWS, "resolution": [RES, RES]},
        "cpu_baseline": {"value": value, "unit": "views/s", "kind": "reference", "cores": 1,
                         "sample": "full step; the reference's own CUDA kernels (renderer, EG, camera projection, "
                                   "mesh boundary, silhouette loss; unmodified, sm_100a) launched per op like its TF "
                                   "ops (renderer per frame), Pose2EG on the host (numpy restatement of the C++ op), "
                                   "losses as torch elementwise ops"},
        "e2e": {"value": value, "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--frames", type=int, default=FRAMES, help="frames per rank (default 16; smaller for profiling)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default raster tiling (8 px, 256)")
    args = ap.parse_args()
    globals()["FRAMES"] = args.frames
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else max(args.warmup, 1)
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        D.finalize(world)


if __name__ == "__main__":
    main()
