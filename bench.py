#!/usr/bin/env python
"""Benchmark of the deform-and-render chain: fwd+bwd views/s at 81,920 triangles, 1024x1024.

Workload (one "step"): 16 frames x 8 views of an icosphere subdivision-6 mesh
(40,962 vertices / 81,920 triangles, radius 1 m = 1000 units, 1 cm vertex
jitter), cameras on a 3 m ring (fx = fy = 1200), vertex-colour rasterization,
the masked L1 image loss against seeded target images, and the renderer
adjoint (gradients w.r.t. vertex positions and vertex colours).  Synthetic
data; inputs larger than L2 (1.6 GB of target images per step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

ours:       the chain through libhc.so, captured once in a CUDA graph and
            replayed (value: device time, inputs resident in HBM); e2e runs the
            same step through the public Python API with every step's inputs
            copied from pinned host memory and the loss read back.
reference:  the reference's own CUDA kernels (compiled unmodified for sm_100a
            into oracle/_ref) driven per frame like its TF ops, the plain
            per-view per-op path, with the L1 loss as elementwise torch ops.
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
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        torch.distributed.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    t = torch.tensor([x], device="cuda", dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------------
# workload
# --------------------------------------------------------------------------
def make_workload(rank: int):
    from deepcharacters_b200 import synthetic as S
    sc = S.render_scene(SUBDIV, batch=FRAMES, views=VIEWS, width=RES, height=RES, seed=2 + 100 * rank, fx=1200.0,
                        texture_size=16)
    # the foreground mask of the data term: inside of a seeded ellipse per view
    return sc


def cpu_baseline(sc, frames=1, views=2):
    """The oracle restatement in float on the host cores (bounded sample)."""
    from oracle import oracle as O
    sub = {k: sc[k] for k in ("faces", "texcoords")}
    B, C = frames, views
    verts = sc["verts"][:B]
    colors = sc["colors"][:B]
    extr = sc["extr"][:B, :12 * C]
    intr = sc["intr"][:B, :9 * C]
    sh = sc["sh"][:B, :C]
    target = sc["target"][:B, :C]
    tex = sc["texture"][:B]
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    fw = O.render_forward(sub["faces"], sub["texcoords"], B, C, RES, RES, "vertexColor", "shadeless", verts, colors,
                          tex, sh, extr, intr, precision="f32", nthreads=cores, fragile=False)
    m = (fw["face"] >= 0)[..., None]
    diff = 255.0 * (fw["render"] - target) * m
    cnt = max(int(np.count_nonzero(diff)), 1)
    g = (255.0 * np.sign(diff) / cnt).astype(np.float32)
    O.render_backward(sub["faces"], sub["texcoords"], B, C, RES, RES, "vertexColor", "shadeless", g, verts, colors,
                      tex, sh, target, fw["vnormal"], fw["bary"], fw["face"], extr, intr, precision="f32",
                      nthreads=cores)
    dt = time.perf_counter() - t0
    return {"value": B * C / dt, "unit": "views/s", "cores": cores, "kind": "port",
            "sample": f"{B} frame x {C} views of the same workload (fwd + L1 + bwd, float oracle, OpenMP)"}


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
class Chain:
    """One fwd + loss + bwd step through libhc.so on device-resident buffers."""

    def __init__(self, sc, dev):
        from deepcharacters_b200.renderer import RendererEngine
        self.eng = RendererEngine(sc["faces"], sc["texcoords"], sc["N"], VIEWS, RES, RES, "vertexColor", "shadeless",
                                  2, 2)
        self.eng.set_tuning(8, 256)
        self.eng.reserve(FRAMES)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        self.inp = {k: t(sc[k]) for k in ("verts", "colors", "texture", "sh", "extr", "intr", "target")}
        B, C, H, W, N = FRAMES, VIEWS, RES, RES, sc["N"]
        self.out = dict(bary=torch.empty((B, C, H, W, 2), device=dev), face=torch.empty((B, C, H, W), device=dev,
                                                                                         dtype=torch.int32),
                        render=torch.empty((B, C, H, W, 3), device=dev), vnormal=torch.empty((B, C, N, 3), device=dev))
        self.grad_img = torch.empty((B, C, H, W, 3), device=dev)
        self.loss = torch.zeros((1,), device=dev)
        self.ws = torch.zeros((4,), device=dev, dtype=torch.float64)
        self.gpos = torch.empty((B, N, 3), device=dev)
        self.gcol = torch.empty((B, N, 3), device=dev)
        self.gsh = torch.empty((B, C, 27), device=dev)
        self.n_px = B * C * H * W

    def forward(self):
        i = self.inp
        self.eng.forward(i["verts"], i["colors"], i["texture"], i["sh"], i["extr"], i["intr"], out=self.out)

    def loss_grad(self):
        from deepcharacters_b200 import _lib
        from deepcharacters_b200.renderer import _stream
        P = _lib.ptr
        _lib.call("hc_image_l1_loss", _stream(), self.n_px, P(self.out["render"]), P(self.inp["target"]),
                  P(self.out["face"]), None, P(self.ws), P(self.loss), P(self.grad_img))

    def backward(self):
        from deepcharacters_b200 import _lib
        from deepcharacters_b200.renderer import _stream
        P = _lib.ptr
        i, o = self.inp, self.out
        _lib.call("hc_renderer_backward", self.eng.handle, _stream(), FRAMES, P(self.grad_img), P(i["verts"]),
                  P(i["colors"]), P(i["texture"]), 16, 16, P(i["sh"]), P(i["target"]), P(o["vnormal"]),
                  P(o["bary"]), P(o["face"]), P(i["extr"]), P(i["intr"]), P(self.gpos), P(self.gcol), None,
                  P(self.gsh))

    def step(self):
        self.forward()
        self.loss_grad()
        self.backward()


def run_ours(args, world, rank, local):
    from deepcharacters_b200 import _lib
    dev = torch.device("cuda", local)
    sc = make_workload(rank)
    ch = Chain(sc, dev)
    views_per_step = FRAMES * VIEWS
    # eager warm-up (allocates every workspace), then capture one step
    for _ in range(2):
        ch.step()
    torch.cuda.synchronize()
    l0 = _lib.lib().hc_kernel_launches()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            ch.step()
    launches_per_step = _lib.lib().hc_kernel_launches() - l0
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()

    def allreduce():
        if world > 1:
            torch.distributed.all_reduce(ch.gcol)

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
    for name, fn in (("render_forward", ch.forward), ("image_l1_loss", ch.loss_grad),
                     ("render_backward", ch.backward)):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(3):
            fn()
        b.record()
        torch.cuda.synchronize()
        stage_ms[name] = a.elapsed_time(b) / 3
    N, F = sc["N"], sc["F"]
    P = RES * RES
    stage_bytes = {  # algorithmic bytes per call
        "render_forward": views_per_step * 24 * P + FRAMES * (24 * N + 12 * F),
        "image_l1_loss": views_per_step * (12 + 12 + 4 + 12) * P,
        "render_backward": views_per_step * (4 + 8 + 12 + 12) * P + FRAMES * (24 * N + 12 * F + 24 * N),
    }
    dom = max(stage_ms, key=stage_ms.get)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    ach = stage_bytes[dom] / (stage_ms[dom] / 1e3) / 1e9
    traffic_path = os.path.join(ROOT, "profiles", "traffic.json")
    traffic = None
    if os.path.exists(traffic_path):
        traffic = json.load(open(traffic_path)).get(dom)

    # e2e: public API, pinned host inputs copied every step, loss read back
    e2e = None if args.no_e2e else run_e2e(ch, sc, dev, args, world)

    line = {
        "metric": METRIC, "value": value, "unit": "views/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded icosphere, ring cameras, random targets)",
        "config": {"workload": "icosphere subdiv-6 (40,962 verts / 81,920 tris) x 16 frames x 8 views 1024x1024, "
                               "vertexColor shadeless raster + masked L1 + adjoint, CUDA graph",
                   "frames": FRAMES, "views": VIEWS, "resolution": [RES, RES], "triangles": F,
                   "parallelism": f"frames sharded, {world} rank(s)",
                   "l2": "inputs larger than L2 (1.6 GB of target images per step)",
                   "raster_tile": 8, "bin_capacity": 256},
        "e2e": e2e,
        "gpu_launches": int(launches_per_step * args.steps),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650",
                     "stage_ms": stage_ms,
                     "chain_bytes_per_view": algorithmic_bytes_per_view(N, F, RES, RES, VIEWS),
                     "chain_frac": algorithmic_bytes_per_view(N, F, RES, RES, VIEWS) * value / world / 1e9 / peak},
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sc)
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_e2e(ch, sc, dev, args, world):
    """Same step through the public API with host inputs: per step H2D of
    vertex positions, colours, cameras, SH and target images from pinned
    memory (double-buffered on a copy stream) and D2H of the loss."""
    keys = ("verts", "colors", "sh", "extr", "intr", "target")
    host = {k: torch.from_numpy(np.ascontiguousarray(sc[k])).pin_memory() for k in keys}
    bufs = [{k: torch.empty_like(ch.inp[k]) for k in keys} for _ in range(2)]
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    copy = torch.cuda.Stream()
    loss_host = torch.zeros((1,), dtype=torch.float32).pin_memory()
    ready = [torch.cuda.Event() for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]
    saved = dict(ch.inp)

    def upload(slot):
        with torch.cuda.stream(copy):
            copy.wait_event(done[slot])
            for k in keys:
                bufs[slot][k].copy_(host[k], non_blocking=True)
            ready[slot].record(copy)

    def run(n):
        for i in range(2):
            done[i].record()
        upload(0)
        for i in range(n):
            slot = i % 2
            torch.cuda.current_stream().wait_event(ready[slot])
            if i + 1 < n:
                upload((i + 1) % 2)
            for k in keys:
                ch.inp[k] = bufs[slot][k]
            ch.step()
            if world > 1:
                torch.distributed.all_reduce(ch.gcol)
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
            "d2h_bytes_per_step": 4, "ms_per_step": dt / args.steps * 1e3,
            "path": "RendererEngine.forward + hc_image_l1_loss + hc_renderer_backward, eager, pinned double buffer"}


# --------------------------------------------------------------------------
# reference arm
# --------------------------------------------------------------------------
def run_reference(args, world, rank, local):
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhcref.so was not built"}))
        return
    dev = torch.device("cuda", local)
    sc = make_workload(0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    inp = {k: t(sc[k]) for k in ("verts", "colors", "texture", "sh", "extr", "intr", "target")}
    ref = O.RefRenderer(sc["faces"], sc["texcoords"], sc["N"], VIEWS, RES, RES, "vertexColor", "shadeless", "none", 2,
                        2)

    def step():
        fw = ref.forward(FRAMES, inp["verts"], inp["colors"], inp["texture"], inp["sh"], inp["extr"], inp["intr"],
                         depth=False, sync_each=0)
        diff = 255.0 * (fw["render"] - inp["target"]) * (fw["face"] >= 0).unsqueeze(-1)
        cnt = torch.count_nonzero(diff).clamp_min(1)
        g = 255.0 * torch.sign(diff) / cnt
        ref.backward(FRAMES, g.contiguous(), inp["verts"], inp["colors"], inp["texture"], inp["sh"], inp["target"],
                     fw["vnormal"], fw["bary"], fw["face"], inp["extr"], inp["intr"])

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
        "config": {"workload": "icosphere subdiv-6 (40,962 verts / 81,920 tris) x 16 frames x 8 views 1024x1024, "
                               "vertexColor shadeless raster + masked L1 + adjoint",
                   "frames": FRAMES, "views": VIEWS, "resolution": [RES, RES]},
        "cpu_baseline": {"value": value, "unit": "views/s", "kind": "reference", "cores": 1,
                         "sample": "full step; the reference's own CUDA kernels (CUDABasedRasterization{,Grad}.cu, "
                                   "unmodified, sm_100a) launched per frame from one host thread like its TF ops"},
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
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
