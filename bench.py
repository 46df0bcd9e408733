#!/usr/bin/env python
"""Benchmark of the deform-and-render chain: fwd+bwd views/s at 81,920 triangles, 1024x1024.

Workload (one "step"): the deform-and-render chain on 16 frames x 8 views of
a character built on an icosphere subdivision-6 mesh (40,962 vertices /
81,920 triangles, radius 1 m = 1000 units, 1 cm vertex jitter): node skinning
of a 1000-node embedded graph by a 24-joint tree (3 revolute dofs each),
embedded-graph deformation, vertex-colour rasterization at 1024x1024 from
cameras on a 3 m ring (fx = fy = 1200), the masked L1 image loss, camera
projection + projected-mesh boundary + the silhouette distance-transform loss,
and the adjoints back to node rotations / translations, joint angles and
vertex colours.  Synthetic data; inputs larger than L2 (1.6 GB of target
images per step).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--adjoint parity|exact]

ours:       the chain through libhc.so, captured once in a CUDA graph and
            replayed (value: device time, inputs resident in HBM); e2e runs the
            same step through the public Python API with every step's inputs
            copied from pinned host memory and the loss read back; `unbatched`
            runs the same kernels one view per call, eagerly, without a graph.
            The renderer adjoint is the reference's barycentric-Jacobian
            formula (`parity`, the mode checked against the reference kernels
            at this shape) unless `--adjoint exact` selects the closed form.
reference:  the reference's own CUDA kernels (compiled unmodified for sm_100a
            into oracle/_ref) driven op by op like its TF ops (the renderer
            per frame), node skinning on the host as the reference's CPU op,
            the losses as elementwise torch ops: the plain per-op path.
With N > 1 every rank renders its own 16 frames (weak scaling; frames
sharded by ``dist.rank_frames``) and the gradient of the shared vertex
colours is summed over frames and ranks (NCCL all-reduce) every step.  Run
bare with --gpus N > 1, the script starts the N ranks itself.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
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
SEED = 2
WORKLOAD = ("deform-and-render chain fwd+bwd: icosphere subdiv-6 (40,962 verts / 81,920 tris), 1000-node embedded "
            "graph (K=4) skinned by a 24-joint tree (72 revolute dofs, node DQ), 16 frames x 8 views 1024x1024, "
            "vertexColor raster + masked L1 + silhouette DT loss, gradients to node rotations / translations, joint "
            "angles and vertex colours")


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
    """SM clock and clock-event reasons of this rank's GPU sampled every
    20 ms during the timed region (NVML; nvidia-smi at 200 ms if NVML is
    unavailable)."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, cuda_index: int, period_s: float = 0.02):
        self.cuda_index = cuda_index
        self.period = period_s
        self.samples = []  # (sm_mhz, max_mhz, reason names, power W)
        self.stop_evt = threading.Event()
        self.thread = None
        self.source = None
        self.proc = None

    def _nvml_handle(self):
        import pynvml as N
        N.nvmlInit()
        p = torch.cuda.get_device_properties(self.cuda_index)
        try:
            bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
            return N, N.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return N, N.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def _nvml_loop(self, N, h):
        get_reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            N.nvmlDeviceGetCurrentClocksThrottleReasons
        masks = [(name, getattr(N, attr, 0)) for name, attr in self.REASONS]
        mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        while not self.stop_evt.is_set():
            try:
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                r = get_reasons(h)
                pw = N.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.samples.append((float(sm), float(mx), [n for n, m in masks if m and (r & m)], pw))
            except Exception:
                pass
            self.stop_evt.wait(self.period)

    def start(self):
        try:
            N, h = self._nvml_handle()
            self.source = "nvml"
            self.thread = threading.Thread(target=self._nvml_loop, args=(N, h), daemon=True)
            self.thread.start()
            return
        except Exception:
            pass
        fields = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                  "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                  "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.cuda_index), f"--query-gpu={fields}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            return
        self.source = "nvidia-smi"

        def read():
            names = [n for n, _ in self.REASONS[:4]]
            for line in self.proc.stdout:
                r = [x.strip() for x in line.split(",")]
                try:
                    self.samples.append((float(r[0]), float(r[1]),
                                         [n for n, x in zip(names, r[3:7]) if x.lower().startswith("active")],
                                         float(r[2])))
                except (ValueError, IndexError):
                    pass

        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()

    def stop(self):
        self.stop_evt.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"], "samples": 0}
        reasons = sorted({n for _, _, rs, _ in self.samples for n in rs})
        return {"sm_mhz": statistics.median(x[0] for x in self.samples),
                "sm_max_mhz": max(x[1] for x in self.samples), "reasons": reasons, "samples": len(self.samples),
                "power_w_max": max(x[3] for x in self.samples), "source": self.source}


# --------------------------------------------------------------------------
# distributed plumbing
# --------------------------------------------------------------------------
def dist_setup(gpus: int):
    world, rank, local = D.env_rank()
    if world != gpus:
        raise SystemExit(f"bench.py: --gpus {gpus} but WORLD_SIZE={world} ranks were launched")
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


def make_workload(first: int, count: int):
    """Frames first .. first+count-1 of the job's seeded sequence (one
    character, per-frame poses / node deltas / lighting / targets)."""
    from deepcharacters_b200 import synthetic as S
    return S.chain_scene(SUBDIV, N_NODES, N_SKEL, count, VIEWS, RES, RES, seed=SEED, fx=FX, first_frame=first)


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
                      "adjoint + EG adjoint (float oracle built -O3 -fopenmp, OpenMP over all host threads; "
                      "silhouette terms not in the sample)"}


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------
def stage_bytes(sc, frames):
    """Algorithmic bytes per call of each stage (compulsory traffic of what
    the stage must read and write once)."""
    B, C, P, N, F, M = frames, VIEWS, RES * RES, sc["N"], sc["F"], sc["M"]
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


def kernel_bytes(sc, frames, covered):
    """Algorithmic bytes per launch of the two raster kernels over frames x
    VIEWS views with the image L1 fused in (``covered`` = pixels with a face,
    all views).  k_resolve writes face 4 + barycentrics 8 + colour 12 B for
    every pixel (background included: the buffers are outputs), reads the
    target (12 B) of the covered pixels and each frame's positions, colours
    and faces once.  k_render_grad reads the face id (4 B) of every pixel and,
    of the covered pixels only, the render 12 (the image gradient is formed
    from it), the barycentrics 8 and the target 12 B, plus each frame's
    positions, colours and faces, and writes the position and colour
    gradients."""
    V, P, N, F = frames * VIEWS, RES * RES, sc["N"], sc["F"]
    return {"resolve": V * 24 * P + 12 * covered + frames * (24 * N + 12 * F),
            "render_grad": V * 4 * P + 32 * covered + frames * (24 * N + 12 * F + 24 * N)}


def issue_roofline(kern_ms, views, clocks, device, adjoint="parity"):
    """Instruction-issue ceiling of the two raster kernels (they are
    issue-bound, not HBM-bound): ncu's warp instructions per view of each
    (profiles/issue.json, a small capture of the same kernels; the count
    grows with the views rendered) x the views of this launch / the live
    kernel time, against the SMs' issue rate (4 warp instructions per SM per
    clock) at the SM clock sampled during the timed region."""
    path = os.path.join(ROOT, "profiles", "issue.json")
    if not os.path.exists(path):
        return {}
    ij = json.load(open(path))
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    peak = sms * 4 * mhz * 1e6 / 1e9  # G warp instructions / s
    out = {"issue_peak_ginst_s": peak, "issue_peak_basis": f"{sms} SMs x 4 warp inst/clk x {mhz:.0f} MHz"}
    for k, ms in kern_ms.items():
        rec = ij.get("k_" + k + ("_exact" if k == "render_grad" and adjoint == "exact" else ""))
        if not rec:
            continue
        ach = rec["warp_inst_per_view"] * views / (ms / 1e3) / 1e9
        out[k] = {"achieved_ginst_s": ach, "frac": ach / peak, "lanes_per_inst": rec["lanes_per_inst"],
                  "warp_inst_per_view": rec["warp_inst_per_view"], "capture": rec.get("capture")}
    return out


def one_view_scene(sc):
    """The scene arrays of frame 0, camera 0 (shapes of a 1-frame 1-view chain)."""
    d = dict(sc)
    for k in ("dofs", "dT", "dA", "disp", "colors", "texture"):
        d[k] = sc[k][:1]
    for k in ("sh", "target", "target_u8", "dt", "crops"):
        d[k] = sc[k][:1, :1]
    d["extr"], d["intr"] = sc["extr"][:1, :12], sc["intr"][:1, :9]
    return d


def view_inputs(inp, f, c):
    """Views into a batched chain's input tensors: frame f, camera c."""
    o = {k: inp[k][f:f + 1] for k in ("dofs", "dT", "dA", "disp", "colors", "texture")}
    o.update({k: inp[k][f:f + 1, c:c + 1] for k in ("sh", "target", "dt", "crops")})
    o["extr"], o["intr"] = inp["extr"][f:f + 1, 12 * c:12 * c + 12], inp["intr"][f:f + 1, 9 * c:9 * c + 9]
    return o


def run_unbatched(ch, sc, dev, frames, parity, steps):
    """The same kernels without batching or graph capture: one chain call
    per (frame, view), eager (node skinning, EG, raster + L1, silhouette and
    all adjoints per view), the raster tiling of the batched chain."""
    from deepcharacters_b200.chain import DeformRenderChain
    one = DeformRenderChain(one_view_scene(sc), dev, 1, 1, RES, RES, W_SIL, W_SIL1, tile=ch.tuning[0],
                            bin_capacity=ch.tuning[1], gradient_parity=parity)
    pairs = [(f, c) for f in range(frames) for c in range(VIEWS)]

    def step():
        for f, c in pairs:
            one.inp.update(view_inputs(ch.inp, f, c))
            one.step()

    step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        step()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    return {"value": len(pairs) / (ms / 1e3), "unit": "views/s", "ms_per_step": ms, "steps": steps,
            "how": "the same libhc kernels issued one view per call (a 1-frame, 1-camera DeformRenderChain stepped "
                   "eagerly over every (frame, view) of the step: node skinning, EG, raster + L1, silhouette and "
                   "all adjoints per view), no CUDA graph; device time (CUDA events)"}


def parity_record(adjoint):
    """The committed record of tests/test_chain_c2_gpu.py (the chain at this
    per-frame shape, 1 frame x 4 views, against the reference kernels and the
    FP64 oracle), quoted for the adjoint mode this run times."""
    path = os.path.join(ROOT, "profiles", "parity_c2.json")
    if not os.path.exists(path):
        return {"adjoint": adjoint, "record": None}
    rec = json.load(open(path))
    out = {"adjoint": adjoint, "record": "profiles/parity_c2.json (tests/test_chain_c2_gpu.py on a B200)"}
    ref = rec.get("parity_mode_vs_reference_kernels", {})
    f64 = rec.get("adjoints_vs_fp64", {})
    if adjoint == "parity":
        out["vs_reference_kernels"] = {k: ref[k] for k in ("loss", "gv", "gcol", "gT", "gA", "gv_sil",
                                                           "face_mismatch_outside_ties", "tie_pixels") if k in ref}
    mode = f64.get(adjoint, {})
    out["vs_fp64"] = {px: {k: v for k, v in mode.get(px, {}).items()}
                      for px in ("all_pixels", "well_conditioned_pixels") if px in mode}
    if "joint_angles_vs_fp64_central_differences" in f64:
        out["vs_fp64"]["joint_angles_central_differences"] = f64["joint_angles_vs_fp64_central_differences"]
    return out


def run_ours(args, world, rank, local):
    from deepcharacters_b200 import _lib
    dev = torch.device("cuda", local)
    from deepcharacters_b200.chain import DeformRenderChain
    first, frames = D.rank_frames(FRAMES, world, rank)
    sc = make_workload(first, frames)
    parity = args.adjoint == "parity"
    ch = DeformRenderChain(sc, dev, frames, VIEWS, RES, RES, W_SIL, W_SIL1, gradient_parity=parity)
    views_per_step = frames * VIEWS
    gcol_shared = torch.zeros((sc["N"], 3), device=dev)
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

    def reduce_shared():  # the vertex colours are one parameter of every frame and rank
        D.shared_gradient(ch.buf["gcol"], gcol_shared, world)

    for _ in range(args.warmup):
        g.replay()
        reduce_shared()
    torch.cuda.synchronize()
    barrier(world)
    clk = ClockSampler(local)
    clk.start()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    st.record()
    for _ in range(args.steps):
        g.replay()
        reduce_shared()
    en.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ch.rend.stats()  # raises if a raster capacity overflowed or an adjoint copy failed
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
    sbytes = stage_bytes(sc, frames)
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
    covered = int((ch.buf["face"] >= 0).sum())
    kbytes = kernel_bytes(sc, frames, covered)
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
        tj = json.load(open(traffic_path)).get("k_" + dom + ("_exact" if dom == "render_grad" and args.adjoint == "exact"
                                                            else ""))
        if tj:  # ncu DRAM bytes per view of a smaller capture, scaled to this launch's views
            traffic = tj["dram_bytes_per_view"] * frames * VIEWS
    # issue-rate view of the tile resolve: pixels resolved and bin entries
    # scanned per second (its ceiling is the SMs' instruction issue, not HBM)
    issue = {"resolve_pixels_per_s": frames * VIEWS * RES * RES / (kern_ms["resolve"] / 1e3),
             "resolve_bin_entries_per_s": binned / (kern_ms["resolve"] / 1e3),
             "bin_entries_per_covered_pixel": binned / max(covered, 1)}
    issue.update(issue_roofline(kern_ms, frames * VIEWS, clocks, local, args.adjoint))

    unbatched = None if args.no_unbatched or world > 1 else run_unbatched(ch, sc, dev, frames, parity, 2)
    # e2e: public API, pinned host inputs copied every step, losses read back
    e2e = None if args.no_e2e else run_e2e(ch, sc, dev, args, world, reduce_shared)

    line = {
        "metric": METRIC, "value": value, "unit": "views/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded icosphere character, random pose / node deltas, ring cameras, random targets, "
                "ellipse silhouettes)",
        "config": {"workload": WORKLOAD + ", one CUDA graph per step",
                   "frames": FRAMES, "views": VIEWS, "resolution": [RES, RES], "triangles": F, "vertices": N,
                   "nodes": N_NODES, "joints": 3 * N_SKEL, "adjoint": args.adjoint,
                   "parallelism": f"frames sharded (dist.rank_frames), {world} rank(s), {FRAMES} frames per rank",
                   "l2": "inputs larger than L2 (1.6 GB of target images per step)",
                   "raster_tile": ch.tuning[0], "bin_capacity": ch.tuning[1],
                   "autotune_ms": {f"{t}x{c}": round(v, 3) for (t, c), v in tune.items()},
                   "bin_pairs": binned, "spilled_pairs": spilled},
        "e2e": e2e,
        "unbatched": unbatched,
        "parity": parity_record(args.adjoint),
        "gpu_launches": int(launches_per_step * args.steps),
        "roofline": {"bound": "hbm", "kernel": "k_" + dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks
                     else "fallback 6650",
                     "kernel_ms": kern_ms, "kernel_bytes": kbytes, "covered_pixels": covered,
                     "issue": issue,
                     "stage_ms": stage_ms, "stage_bytes": sbytes,
                     "chain_bytes_per_view": algorithmic_bytes_per_view(N, F, RES, RES, VIEWS),
                     "chain_frac": algorithmic_bytes_per_view(N, F, RES, RES, VIEWS) * value / world / 1e9 / peak},
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(sc)
    if rank == 0:
        print(json.dumps(line), flush=True)


C3_METRIC = ("fwd+bwd views/s at 20,480 tris, 16 frames x 8 views of mixed resolution "
             "{512², 768x1024, 1024², 1536x1024}: one call per stage, one CUDA graph per step")
C3_SUBDIV = 5


def run_ours_c3(args, world, rank, local):
    """The batched mixed-resolution configuration: the subdivision-5 character
    (10,242 vertices / 20,480 triangles) skinned per vertex by dual
    quaternions of a 24-joint tree (U(-0.5, 0.5) joint angles), 16 frames x 8
    cameras whose sizes are drawn uniformly from {512x512, 768x1024,
    1024x1024, 1536x1024} (fx = fy = 600 min(W, H) / 512), vertex-colour
    raster + masked L1 + silhouette DT loss, adjoints to the joint angles and
    vertex colours; every stage one call over all views of the step, the step
    one CUDA graph, the raster tiling autotuned."""
    from deepcharacters_b200 import _lib
    from deepcharacters_b200 import synthetic as S
    from deepcharacters_b200.chain import DeformRenderChain
    dev = torch.device("cuda", local)
    first, frames = D.rank_frames(FRAMES, world, rank)
    ws, hs = S.mixed_camera_sizes(VIEWS, SEED)
    sc = S.chain_scene(C3_SUBDIV, 200, N_SKEL, frames, VIEWS, ws, hs, seed=SEED, first_frame=first)
    parity = args.adjoint == "parity"
    ch = DeformRenderChain(sc, dev, frames, VIEWS, ws, hs, W_SIL, W_SIL1, gradient_parity=parity, deformation="dq")
    gcol_shared = torch.zeros((sc["N"], 3), device=dev)
    tune = ch.autotune() if not args.no_autotune else {}
    binned, spilled = ch.check()
    for _ in range(2):
        ch.step()
    torch.cuda.synchronize()
    l0 = _lib.lib().hc_kernel_launches()
    g = ch.capture_step()
    launches_per_step = _lib.lib().hc_kernel_launches() - l0

    def reduce_shared():
        D.shared_gradient(ch.buf["gcol"], gcol_shared, world)

    for _ in range(args.warmup):
        g.replay()
        reduce_shared()
    torch.cuda.synchronize()
    barrier(world)
    clk = ClockSampler(local)
    clk.start()
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record()
    for _ in range(args.steps):
        g.replay()
        reduce_shared()
    en.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ch.rend.stats()  # raises if a raster capacity overflowed or an adjoint copy failed
    ms = max_over_ranks(st.elapsed_time(en) / args.steps, world)
    barrier(world)
    value = frames * VIEWS * world / (ms / 1e3)
    ch.rend.set_kernel_timing(True)
    kern = {}
    for _ in range(3):
        ch.forward()
        ch.backward()
        for k, v in ch.rend.kernel_times().items():
            kern.setdefault(k, []).append(v)
    ch.rend.set_kernel_timing(False)
    kern = {k: sum(v) / len(v) for k, v in kern.items()}
    covered = int((ch.buf["face"] >= 0).sum())
    N, F, P = sc["N"], sc["F"], sc["P_frame"]
    kbytes = {"resolve": frames * 24 * P + 12 * covered + frames * (24 * N + 12 * F),
              "render_grad": frames * 4 * P + 32 * covered + frames * (24 * N + 12 * F + 24 * N)}
    dom = max(("resolve", "render_grad"), key=lambda k: kern[k])
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    ach = kbytes[dom] / (kern[dom] / 1e3) / 1e9
    e2e = None if args.no_e2e else run_e2e(ch, sc, dev, args, world, reduce_shared)
    line = {
        "metric": C3_METRIC, "value": value, "unit": "views/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded icosphere character, random poses, ring cameras of mixed sizes, "
                                "random targets, ellipse silhouettes)",
        "config": {"workload": "batched mixed-resolution chain fwd+bwd: icosphere subdiv-5 (10,242 verts / 20,480 "
                               "tris), vertex DQ skinning by a 24-joint tree (72 revolute dofs), 16 frames x 8 views "
                               "at per-camera sizes drawn from {512x512, 768x1024, 1024x1024, 1536x1024}, "
                               "vertexColor raster + masked L1 + silhouette DT loss, gradients to joint angles and "
                               "vertex colours, one CUDA graph per step",
                   "frames": FRAMES, "views": VIEWS, "camera_sizes": [[w, h] for w, h in zip(ws, hs)],
                   "pixels_per_frame": P, "triangles": F, "vertices": N, "joints": 3 * N_SKEL,
                   "adjoint": args.adjoint, "parallelism": f"frames sharded, {world} rank(s)",
                   "l2": "inputs larger than L2 (%.0f MB of target images per step)" % (frames * P * 12 / 1e6),
                   "raster_tile": ch.tuning[0], "bin_capacity": ch.tuning[1],
                   "autotune_ms": {f"{t}x{c}": round(v, 3) for (t, c), v in tune.items()},
                   "bin_pairs": binned, "spilled_pairs": spilled},
        "e2e": e2e,
        "gpu_launches": int(launches_per_step * args.steps),
        "roofline": {"bound": "hbm", "kernel": "k_" + dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "traffic": None,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks
                     else "fallback 6650",
                     "kernel_ms": kern, "kernel_bytes": kbytes, "covered_pixels": covered},
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


E2E_KEYS = ("dofs", "dT", "dA", "colors", "sh", "extr", "intr", "target_u8", "dt")


def run_e2e(ch, sc, dev, args, world, reduce_shared):
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
            reduce_shared()
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
    return {"value": ch.B * VIEWS * world * args.steps / dt, "unit": "views/s", "h2d_bytes_per_step": h2d,
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
    sc = make_workload(0, FRAMES)
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
        "config": {"workload": WORKLOAD, "frames": FRAMES, "views": VIEWS, "resolution": [RES, RES]},
        "cpu_baseline": {"value": value, "unit": "views/s", "kind": "reference", "cores": 1,
                         "sample": "full step; the reference's own CUDA kernels (renderer, EG, camera projection, "
                                   "mesh boundary, silhouette loss; unmodified, sm_100a) launched per op like its TF "
                                   "ops (renderer per frame), Pose2EG on the host (numpy restatement of the C++ op), "
                                   "losses as torch elementwise ops"},
        "e2e": {"value": value, "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 150 for ours, about 3 s; 10 for the reference arm)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--adjoint", choices=("parity", "exact"), default="parity",
                    help="renderer adjoint: the reference's barycentric-Jacobian formula (parity) or the closed form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-unbatched", action="store_true", help="skip the un-batched, no-graph leg")
    ap.add_argument("--frames", type=int, default=FRAMES, help="frames per rank (default 16; smaller for profiling)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default raster tiling (8 px, 256)")
    ap.add_argument("--config", choices=("c2", "c3"), default="c2",
                    help="c2: the headline chain (default); c3: the batched mixed-resolution chain (own line)")
    args = ap.parse_args(argv)
    if args.steps is None:
        args.steps = 150 if args.impl == "ours" else 10
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else max(args.warmup, 1)
    return args


def run(args):
    globals()["FRAMES"] = args.frames
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            if args.config != "c2":
                if rank == 0:
                    print(json.dumps({"impl": "reference", "config": args.config,
                                      "unavailable": "the reference arm is run for the headline configuration only"}))
            else:
                run_reference(args, world, rank, local)
        elif args.config == "c3":
            run_ours_c3(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        D.finalize(world)


def _spawned_rank(rank, world, port, argv):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), LOCAL_WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    run(parse_args(argv))


def main():
    args = parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # started bare: one process per GPU, rendezvous on 127.0.0.1
        import torch.multiprocessing as mp
        if torch.cuda.device_count() < args.gpus:
            raise SystemExit(f"bench.py: --gpus {args.gpus} but {torch.cuda.device_count()} GPUs are visible")
        with socket.socket() as s:
            s.bind(("127.0.0.1", 0))
            port = s.getsockname()[1]
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_spawned_rank, args=(r, args.gpus, port, sys.argv[1:])) for r in range(args.gpus)]
        for p in procs:
            p.start()
        for p in procs:
            p.join()
        sys.exit(max(abs(p.exitcode or 0) for p in procs))
    run(args)


if __name__ == "__main__":
    main()
