#!/usr/bin/env python
"""Forward + adjoint throughput of the beta-surfel renderer on one node.

Workload "box200k" (default): the synthetic box scene with 200k surfels,
8 cameras on a ring of radius 1.5 at 512x512, 16 gather passes and 16
adjoint passes per pixel, depth 6 (photon and adjoint bounces), 1M photons,
gather radius 0.01.  One step = photon pass + photon grid + camera gather of
all views, dL/dI of the L2 image loss against a target render (positions
jittered N(0, 0.005), albedo N(0, 0.05)), adjoint pass of all views with
gradient accumulation, and (N > 1) a sum all-reduce of the gradients.

Metric: Mrays/s = ray segments submitted to scene traversal (photon bounces
+ camera-gather layers + adjoint bounces) per second of the step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # the 200k-surfel, 8-view workload (throughput headline)
    "box200k": dict(n=200000, cams=8, res=512, photons=1000000, bounces=6, forward_passes=1, spp=16,
                    adjoint_bounces=6, adjoint_spp=16, radius=0.01),
    # the 10k-surfel, single-view workload
    "box10k": dict(n=10000, cams=1, res=256, photons=100000, bounces=4, forward_passes=1, spp=4,
                   adjoint_bounces=4, adjoint_spp=4, radius=0.02),
    # the memory-bound case: 1M surfels, 32 views of 800x800, 64 passes, depth 8
    "box1m-32view": dict(n=1000000, cams=32, res=800, photons=1000000, bounces=8, forward_passes=1, spp=64,
                         adjoint_bounces=8, adjoint_spp=64, radius=0.01),
    # box200k's scene and photon map with one 256x256 view and 8 passes: the
    # case the per-kernel profiles are captured on (under 1 GB resident)
    "box200k-1view": dict(n=200000, cams=1, res=256, photons=1000000, bounces=6, forward_passes=1, spp=8,
                          adjoint_bounces=6, adjoint_spp=8, radius=0.01),
}

METRIC = "fwd+adjoint Mrays/s"
L2_POLICY = "GPU arm: a 256 MB buffer (> 126 MB L2) zeroed between timed steps"


def config_for(name: str, w: dict) -> dict:
    """The bench line's config: the workload and the L2 policy, the same in
    both arms."""
    return {"workload": name, **w, "l2": L2_POLICY}


def settings_for(w: dict) -> dict:
    return {"photons": w["photons"], "bounces": w["bounces"], "forward_passes": w["forward_passes"],
            "gather_passes": w["spp"], "adjoint_bounces": w["adjoint_bounces"], "adjoint_passes": w["adjoint_spp"],
            "gather_radius": w["radius"], "seed": 42, "rng_mode": "decorrelated"}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        sm.sort()
        # other processes computing on this GPU would slow every kernel down
        try:
            apps = subprocess.run(["nvidia-smi", f"--id={self.idx}", "--query-compute-apps=pid",
                                   "--format=csv,noheader"], capture_output=True, text=True, timeout=20).stdout
            procs = len([x for x in apps.split() if x.strip()])
        except Exception:
            procs = None
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "compute_processes": procs,
                "samples": len(sm)}


# --------------------------------------------------------------- helpers
# Algorithmic bytes per kernel of one step, from the device counters:
# a ray segment reads/writes 32 + 32 B of ray state and a 16 B hit record,
# 32 B per BVH node visited and 52 B per surfel test; a photon lookup reads
# 36 B per photon scanned and 8 B (two cell offsets) per grid row of its
# window (25 rows); the adjoint bounce also reads and writes its 48 B
# pending state, and its three kernels (mesh pass, persistent walk,
# shading) pass 128 B of hit and walk records per ray between them (written
# 64 B, read 48 + 16 B); a gradient event is a 64 B record, its lookup and
# an 8 B atomic read-modify-write.
ROWS_PER_QUERY = 25
FWD_COUNTERS = ("photon_segments", "photons_stored", "gather_segments", "gather_node_visits", "gather_surfel_tests",
                "gather_queries", "gather_photons_scanned")
ADJ_COUNTERS = ("adjoint_segments", "node_visits", "surfel_tests", "gradient_events", "gather_queries",
                "photons_scanned")


def kernel_bytes(sf: dict, sb: dict, estimator: str = "reference", all_grads: bool = False) -> dict:
    seg = lambda segs, nodes, tests: 80.0 * segs + 32.0 * nodes + 52.0 * tests
    look = lambda q, scanned: 36.0 * scanned + 8.0 * ROWS_PER_QUERY * q
    fwd_q = sf["gather_queries"]
    adj_q = sb["gather_queries"]
    out = {
        "k_cg_round": seg(sf["gather_segments"], sf["gather_node_visits"], sf["gather_surfel_tests"]),
        "k_cg_lookup": look(fwd_q, sf["gather_photons_scanned"]),
    }
    if estimator == "gather":
        # the sweep: per path segment its direction, links, radiance (read
        # and written) and dL/dI (96 B); per layer record its two float4s,
        # read twice, the surfel's opacity and albedo, and the gradient
        # atomics (opacity, or 16 terms with alpha_geom's surfel reads)
        per_rec = 64.0 + 32.0 + (64.0 + 64.0 if all_grads else 4.0)
        out["k_vs_sweep"] = 96.0 * sb["vertex_entries"] + per_rec * sb["vertex_records"]
        return out
    out["k_adj_bounce"] = seg(sb["adjoint_segments"], sb["node_visits"], sb["surfel_tests"]) \
        + (96.0 + 128.0) * sb["adjoint_segments"]
    out["k_transport"] = 72.0 * sb["gradient_events"] + look(adj_q, sb["photons_scanned"])
    return out


def kernel_times(sf: dict, sb: dict, estimator: str = "reference") -> dict:
    out = {"k_cg_round": (sf["trace_ms"], sf["trace_launches"]),
           "k_cg_lookup": (sf["lookup_ms"], sf["lookup_launches"])}
    if estimator == "gather":
        out["k_vs_sweep"] = (sb["transport_ms"], sb["transport_launches"])
    else:
        out["k_adj_bounce"] = (sb["adjoint_bounce_ms"], sb["adjoint_bounce_launches"])
        out["k_transport"] = (sb["transport_ms"], sb["transport_launches"])
    return out


def read_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def read_traffic(kernel: str, launch_ms: float):
    """DRAM bytes of one launch of `kernel`: the DRAM rate of its ncu
    capture on the small case (profiles/traffic.json) times the launch's
    live device time; None without a capture."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        rate = json.load(open(p))[kernel]["dram_bytes_per_s"]
    except Exception:
        return None
    return int(rate * launch_ms / 1e3)


def cpu_reference_run(w: dict, steps: int = 1, warmup: int = 0):
    """The reference's own kernel code on the host cores, on the workload's
    configuration: oracle/_ref/libpale_ref.so (the reference's unmodified
    PrimalKernels.cpp / AdjointKernels.cpp / PostprocessKernel.cpp for the
    CPU, every host thread) on the same scene, cameras, resolution, photon
    count, radius and depths.  A step traces the full photon pass and grid,
    then one gather pass and one adjoint pass of every camera; the
    reference draws one seed per camera for all of its gather passes and
    replays its one adjoint seed in every pass (SyclBridge.cpp:145,
    AdjointKernels.cpp:27, 94), so the other passes of a full step are
    repeats of these, and the step's time and ray count are the photon part
    plus passes x the one-pass parts.  Falls back to the C oracle port when
    the reference's kernels were not built.  Returns (Mrays/s, seconds
    timed, description, kind, steps)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import numpy as np
    from differentiablepointrendering_b200.scene import make_box_scene, make_surfels
    import ref_lib

    threads = os.cpu_count() or 1
    scene = make_box_scene(w["n"], cameras=w["cams"], resolution=w["res"], points=make_surfels(w["n"], 1234))
    st = settings_for(w)
    st.update(gather_passes=1, adjoint_passes=1, rng_mode="reference")
    if ref_lib.available():
        kind = "reference"
        r = ref_lib.ReferenceRenderer(scene, st, threads=threads)
        gather_segments = r.count_gather_segments()
    else:
        from oracle_lib import OracleRenderer
        kind = "port"
        r = OracleRenderer(scene, st, threads=threads)
        gather_segments = None
    total_rays, total_s = 0.0, 0.0
    for k in range(warmup + steps):
        t0 = time.perf_counter()
        img = r.render_forward()
        t1 = time.perf_counter()
        dl = {c: ((img[c][..., :3] - 0.5) / (3 * img[c][..., 0].size)).astype(np.float32)
              for c in scene.camera_names}
        if kind == "reference":
            r.render_backward_opacity(dl)
            t2 = time.perf_counter()
            photon_ms, gather_ms, adjoint_ms = r.times_ms()
            photon_segments, adjoint_segments = r.segments()
            step_s = (photon_ms + w["spp"] * gather_ms + w["adjoint_spp"] * adjoint_ms) / 1e3
            rays = photon_segments + w["spp"] * gather_segments + w["adjoint_spp"] * adjoint_segments
        else:
            sf = r.stats()
            r.render_backward(dl)
            t2 = time.perf_counter()
            sb = r.stats()
            step_s = (sf["photon_ms"] + w["spp"] * sf["gather_ms"] + w["adjoint_spp"] * sb["backward_ms"]) / 1e3
            rays = sf["photon_segments"] + w["spp"] * sf["gather_segments"] + w["adjoint_spp"] * sb["adjoint_segments"]
        if k >= warmup:
            total_rays += rays
            total_s += step_s
    r.close()
    what = "the reference's kernel sources compiled for the CPU" if kind == "reference" else "the C oracle port"
    desc = (f"{what}, {threads} threads, {w['n']} surfels, {w['cams']} cameras at {w['res']}x{w['res']}, "
            f"{w['photons']} photons, depth {w['bounces']}/{w['adjoint_bounces']}, radius {w['radius']}: per step "
            f"the photon pass and grid plus 1 of the {w['spp']} gather and 1 of the {w['adjoint_spp']} adjoint passes "
            f"of every camera, timed; the full step = photon part + passes x one-pass time (the reference repeats "
            f"the same seeds in every pass); {steps} timed steps after {warmup} warm-up")
    return total_rays / total_s / 1e6, total_s, desc, kind, steps


# -------------------------------------------------------------- reference
def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    steps, warmup = max(1, min(args.steps, 3)), min(args.warmup, 1)
    value, secs, desc, kind, ran = cpu_reference_run(w, steps=steps, warmup=warmup)
    line = {"metric": METRIC, "value": round(value, 4), "unit": "Mrays/s", "impl": "reference", "n_gpus": world,
            "steps": ran, "warmup": warmup, "requested_steps": args.steps, "requested_warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_for(args.workload, w),
            "cpu_baseline": {"value": round(value, 4), "unit": "Mrays/s", "cores": os.cpu_count(), "kind": kind,
                             "sample": desc},
            "e2e": {"value": round(value, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- batched
# C4: four box scenes of 50k-500k surfels with cameras on a 16-position ring
# at 256-1024 pixels; an iteration draws 64 views (scene, ring position,
# resolution, passes 1/4/16/32) and runs their forward (with the L2 loss)
# and adjoint.  The batched form renders all 64 views as one camera-gather
# wavefront and one adjoint wavefront over the four scenes (device.ViewBatch),
# each scene tracing its photon map once; the plain forms run one view per
# call (its scene's photon map traced again in every call), and one pass per
# call as the reference's launch loop does (SyclBridge.cpp:136-146, 181-226).
C4 = dict(scenes=(50000, 100000, 250000, 500000), ring=16, resolutions=(256, 512, 768, 1024), spp=(1, 4, 16, 32),
          views=64, photons=1000000, bounces=6, radius=0.01)
C4_TUNE = dict(leaf_size=(1, 2, 4, 8), walk_block=(256, 128, 64), adjoint_batch_paths=(1 << 22, 1 << 20, 1 << 18))


def c4_settings(knobs: dict) -> dict:
    st = {"photons": C4["photons"], "bounces": C4["bounces"], "forward_passes": 1, "gather_passes": max(C4["spp"]),
          "adjoint_bounces": C4["bounces"], "adjoint_passes": max(C4["spp"]), "gather_radius": C4["radius"],
          "seed": 42, "rng_mode": "decorrelated", "camera_seeds": "camera"}
    st.update(knobs)
    return st


def c4_views(rng, count: int):
    nres = len(C4["resolutions"])
    out = []
    for _ in range(count):
        sc = int(rng.integers(len(C4["scenes"])))
        cam = int(rng.integers(C4["ring"])) * nres + int(rng.integers(nres))
        out.append((sc, cam, int(C4["spp"][int(rng.integers(len(C4["spp"])))]), 0))
    return out


class C4Run:
    """The four C4 renderers with one set of knobs, and timed iterations."""

    def __init__(self, knobs: dict, dev):
        from differentiablepointrendering_b200.pale import Renderer
        from differentiablepointrendering_b200.scene import make_box_scene, make_surfels

        self.dev = dev
        self.knobs = dict(knobs)
        st = c4_settings(knobs)
        self.renderers = []
        for n in C4["scenes"]:
            sc = make_box_scene(n, cameras=C4["ring"], resolutions=C4["resolutions"], points=make_surfels(n, 1234))
            self.renderers.append(Renderer.from_scene(sc, st))

    def close(self):
        for r in self.renderers:
            r.close()

    def _event_ms(self, fn, reps: int = 1) -> float:
        import torch

        stream = torch.cuda.current_stream(self.dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    def batched_ms(self, views) -> float:
        import torch
        from differentiablepointrendering_b200.device import ViewBatch

        vb = ViewBatch(self.renderers, views, device=self.dev)
        tgt = torch.zeros(vb.pixels, 3, dtype=torch.float32, device=self.dev)

        def it():
            vb.forward_loss(tgt)
            vb.backward()

        it()   # warm-up (wavefront buffers grow on the first call)
        return self._event_ms(it)

    def plain_ms(self, views, per_pass: bool) -> float:
        import torch
        from differentiablepointrendering_b200.device import ViewBatch

        calls = []
        for sc, cam, spp, depth in views:
            if per_pass:
                one = ViewBatch([self.renderers[sc]], [(0, cam, 1, depth)], device=self.dev)
                calls.append((one, spp))
            else:
                calls.append((ViewBatch([self.renderers[sc]], [(0, cam, spp, depth)], device=self.dev), 1))
        tgts = [torch.zeros(vb.pixels, 3, dtype=torch.float32, device=self.dev) for vb, _ in calls]

        def it():
            for (vb, reps), t in zip(calls, tgts):
                vb.forward_loss(t)                        # the view's photon map, first pass
                for _ in range(reps - 1):
                    vb.forward_loss(t, trace_photons=False)   # further gather passes
                for _ in range(reps):
                    vb.backward()

        calls[0][0].forward_loss(tgts[0])
        calls[0][0].backward()
        return self._event_ms(it)


def c4_measure(dev, tune: bool = True, iterations: int = 1) -> dict:
    """Autotuner + batched and plain C4 iterations.  The autotuner is a
    coordinate descent over the leaf size, the walk block size and the
    adjoint queue depth (adjoint_batch_paths), one batched iteration of a
    16-view sample per candidate; the chosen knobs then time `iterations`
    iterations of 64 drawn views (seed 7) batched, one view per call and one
    pass per call."""
    import numpy as np

    knobs = {"leaf_size": 1, "walk_block": 256, "adjoint_batch_paths": 1 << 24}
    trials = []
    if tune:
        sample = c4_views(np.random.default_rng(3), 16)
        best = None
        for key in ("leaf_size", "walk_block", "adjoint_batch_paths"):
            for v in C4_TUNE[key]:
                cand = dict(knobs, **{key: v})
                run = C4Run(cand, dev)
                try:
                    ms = run.batched_ms(sample)
                finally:
                    run.close()
                trials.append({**cand, "ms": round(ms, 2)})
                if best is None or ms < best[0]:
                    best = (ms, cand)
            knobs = dict(best[1])
    rng = np.random.default_rng(7)
    run = C4Run(knobs, dev)
    try:
        res = {"batched_ms": [], "plain_per_view_ms": [], "plain_per_pass_ms": []}
        for _ in range(iterations):
            views = c4_views(rng, C4["views"])
            res["batched_ms"].append(run.batched_ms(views))
            res["plain_per_view_ms"].append(run.plain_ms(views, per_pass=False))
            res["plain_per_pass_ms"].append(run.plain_ms(views, per_pass=True))
    finally:
        run.close()
    b = float(np.mean(res["batched_ms"]))
    pv = float(np.mean(res["plain_per_view_ms"]))
    pp = float(np.mean(res["plain_per_pass_ms"]))
    return {"workload": "c4", "scenes": list(C4["scenes"]), "views_per_iteration": C4["views"],
            "resolutions": list(C4["resolutions"]), "passes": list(C4["spp"]), "photons": C4["photons"],
            "depth": C4["bounces"], "iterations": iterations, "knobs": knobs, "autotune": trials,
            "batched_iters_per_s": round(1e3 / b, 4), "plain_per_view_iters_per_s": round(1e3 / pv, 4),
            "plain_per_pass_iters_per_s": round(1e3 / pp, 4),
            "speedup_vs_plain_per_view": round(pv / b, 3), "speedup_vs_plain_per_pass": round(pp / b, 3),
            "ms": {"batched": round(b, 2), "plain_per_view": round(pv, 2), "plain_per_pass": round(pp, 2)}}


# ------------------------------------------------------------------- ours
def plain_and_latency(r, frame, target, dev, batched_ms: float, steps: int = 2, requests: int = 20) -> dict:
    """Beside the batched step: (1) the plain path, the same step with one
    view per call (each call traces its photon map and runs its own camera
    gather and adjoint, as render_forward/render_backward per camera do),
    timed with CUDA events; (2) the latency of single-view gradient requests
    (forward + L2 loss + adjoint of camera 0, host-synchronised each), wall
    clock from submission to the result being ready."""
    import numpy as np
    import torch

    from differentiablepointrendering_b200.device import DeviceFrame

    frames, targets, off = [], [], 0
    for i, (w, h) in enumerate(frame.sizes):
        frames.append(DeviceFrame(r, cameras=[frame.cams[i]], device=dev))
        targets.append(target[off:off + w * h].contiguous())
        off += w * h

    def plain_step():
        for f, t in zip(frames, targets):
            f.forward_loss(t)
            f.backward()

    plain_step()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        plain_step()
    b.record(stream)
    torch.cuda.synchronize()
    plain_ms = a.elapsed_time(b) / steps
    lat = []
    for _ in range(requests):
        t0 = time.perf_counter()
        frames[0].forward_loss(targets[0])
        frames[0].backward()
        torch.cuda.synchronize()
        lat.append((time.perf_counter() - t0) * 1e3)
    lat = np.sort(np.array(lat))
    w0, h0 = frame.sizes[0]
    return {
        "plain_per_view": {"ms_per_step": round(plain_ms, 3), "iters_per_s": round(1e3 / plain_ms, 4),
                           "batched_speedup": round(plain_ms / batched_ms, 3), "steps": steps,
                           "note": "same views, passes and seeds settings, one view per forward/adjoint call"},
        "latency_ms": {"request": f"one {w0}x{h0} view: photon pass, gather, L2 loss, adjoint", "n": requests,
                       "p50": round(float(np.percentile(lat, 50)), 3), "p99": round(float(np.percentile(lat, 99)), 3)},
    }


def run_ours(args, rank: int, world: int, local_rank: int):
    import numpy as np
    import torch
    import torch.distributed as dist

    from differentiablepointrendering_b200.build import build_library
    from differentiablepointrendering_b200.device import DeviceFrame
    from differentiablepointrendering_b200.multigpu import reduce_gradients, shard_cameras
    from differentiablepointrendering_b200.pale import Renderer
    from differentiablepointrendering_b200.scene import jitter_target, make_box_scene, make_surfels

    build_library()
    torch.cuda.set_device(local_rank)
    dev = torch.device(f"cuda:{local_rank}")
    w = WORKLOADS[args.workload]
    # weak scaling: one scene with cams x N cameras on the ring, split round
    # robin over the ranks (rank r renders cameras r, r + N, ...: cams each);
    # camera-keyed seeds make a camera's work independent of the split
    st = dict(settings_for(w), camera_seeds="camera", gradients=args.gradients, estimator=args.estimator)
    pts = make_surfels(w["n"], 1234)
    scene = make_box_scene(w["n"], cameras=w["cams"] * world, resolution=w["res"], points=pts)
    mine = shard_cameras(list(range(w["cams"] * world)), rank, world)
    tscene = scene.with_points(jitter_target(pts, 5678))

    # target images (renders of the jittered cloud), resident on the device
    tr = Renderer.from_scene(tscene, st)
    tf = DeviceFrame(tr, cameras=mine, device=dev)
    tf.forward()
    target = tf.ldr[:, :3].clone()
    torch.cuda.synchronize()
    del tf
    tr.close()

    r = Renderer.from_scene(scene, st)
    frame = DeviceFrame(r, cameras=mine, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        frame.forward_loss(target)      # post-process writes dL/dI and the loss
        frame.backward()
        if world > 1:
            reduce_gradients(frame.grads)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    # work per step (fixed seeds: every step traces the same rays)
    frame.forward_loss(target)
    sf = frame.stats()
    frame.backward()
    sb = frame.stats()
    rays = sf["photon_segments"] + sf["gather_segments"] + sb["adjoint_segments"]
    launches = int(sf["kernel_launches"] + sb["kernel_launches"])

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local_rank)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        step()
        ends[k].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    total_rays = torch.tensor([float(rays)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(total_rays)
    ms_per_step = ms / args.steps
    value = float(total_rays.item()) / (ms_per_step / 1e3) / 1e6

    # ---- end to end through the public API with host buffers
    cams = [r.get_camera_names()[i] for i in mine]
    tgt_np = {}
    for i, name in enumerate(cams):
        ww, hh = frame.sizes[i]
        off = sum(a * b for a, b in frame.sizes[:i])
        tgt_np[name] = target[off:off + ww * hh].view(hh, ww, 3).cpu().numpy()
    e2e_steps = max(1, min(args.steps, 3))
    # one untimed step first: the host path's own buffers (the device images,
    # the library's pinned staging of large copies) are allocated on first use
    imgs, dl, losses = r.render_forward_loss(tgt_np)
    r.render_backward(dl)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        imgs, dl, losses = r.render_forward_loss(tgt_np)
        grads, _ = r.render_backward(dl)
        if world > 1:
            for k2, v in grads.items():
                gt = torch.from_numpy(v).to(dev)
                dist.all_reduce(gt)
                grads[k2] = gt.cpu().numpy()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    et = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e_value = float(total_rays.item()) * e2e_steps / float(et.item()) / 1e6
    pix = frame.pixels
    h2d = pix * 12 + pix * 16                  # RGB target; dL/dI (float4 per pixel)
    d2h = 3 * pix * 16 + 8 * len(cams) + r.num_points * 17 * 4   # LDR, raw, dL/dI, losses; gradients

    if rank != 0:
        r.close()
        return
    extra = {} if args.skip_extra else plain_and_latency(r, frame, target, dev, ms_per_step)
    if not args.skip_extra and world == 1:
        r.close()      # frees box200k's buffers for the C4 scenes
        extra["c4"] = c4_measure(dev, tune=not args.no_tune)
    peaks = read_peaks()
    hbm = peaks["hbm_gbs"] if peaks else 6650.0
    # per-kernel device time (events around every launch, stats step) and
    # algorithmic bytes; the roofline entry is the kernel with the most time
    kb = kernel_bytes(sf, sb, args.estimator, args.gradients == "all")
    kt = kernel_times(sf, sb, args.estimator)
    kernels = {}
    for k in kb:
        ms, n = kt[k]
        n = max(1, int(n))
        ach = kb[k] / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        kernels[k] = {"ms_per_step": round(ms, 3), "launches": n, "launch_ms": round(ms / n, 4),
                      "algorithmic_bytes_per_launch": int(kb[k] / n), "achieved_gbs": round(ach, 1),
                      "frac": round(ach / hbm, 4), "dram_bytes_per_launch": read_traffic(k, ms / n)}
    top = max(kernels, key=lambda k: kernels[k]["ms_per_step"])
    achieved = kernels[top]["achieved_gbs"]
    traffic = read_traffic(top, kernels[top]["launch_ms"])
    if args.skip_cpu:
        cpu_val, cpu_desc, cpu_kind = None, "skipped", None
    else:
        cpu_val, _, cpu_desc, cpu_kind, _ = cpu_reference_run(w, steps=1, warmup=0)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_for(args.workload, w),
        "gradients": args.gradients, "estimator": args.estimator,
        "iters_per_s": round(1e3 / ms_per_step, 4), "rays_per_step_per_gpu": int(rays),
        "parallelism": f"{w['cams'] * world} ring cameras split round robin over {world} GPU(s), gradients all-reduced",
        "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps, "warmup": 1},
        "gpu_launches": launches * args.steps,
        "roofline": {"kernel": top, "bound": "hbm", "achieved": round(achieved, 1),
                     "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "traffic": traffic, "peak_source": "measured" if peaks else "fallback",
                     "algorithmic_bytes_per_launch": kernels[top]["algorithmic_bytes_per_launch"],
                     "launch_ms": kernels[top]["launch_ms"], "launches_per_step": kernels[top]["launches"]},
        "kernels": kernels,
        "cpu_baseline": {"value": round(cpu_val, 4) if cpu_val else None, "unit": "Mrays/s",
                         "cores": os.cpu_count(), "kind": cpu_kind, "sample": cpu_desc},
        "clocks": clk,
        "breakdown_ms": {"photon": round(sf["photon_ms"], 3), "gather": round(sf["gather_ms"], 3),
                         "adjoint": round(sb["backward_ms"], 3)},
        # work of one step on this rank (device counters): the units behind
        # the algorithmic bytes of each kernel
        "counters": {"forward": {k: int(sf[k]) for k in FWD_COUNTERS},
                     "adjoint": {k: int(sb[k]) for k in ADJ_COUNTERS}},
        **extra,
    }
    print(json.dumps(line), flush=True)
    if args.skip_extra or world > 1:
        r.close()


# ---------------------------------------------------------------- C3b
C3B_MODES = (   # label, settings
    ("reference adjoint", {"estimator": "reference"}),
    ("gather, checkpoint", {"estimator": "gather", "vertices": "checkpoint"}),
    ("gather, replay", {"estimator": "gather", "vertices": "replay"}),
    ("gather, auto 48 GB", {"estimator": "gather", "vertices": "auto", "vertex_store_bytes": 48 * 10 ** 9}),
)


def run_c3b(args):
    """The memory-bound case: box1m-32view's scene (1M surfels, 32 views of
    800x800, depth 8) at --c3b-passes passes, one forward + backward per
    iteration with all seven gradient groups, for the reference's adjoint
    and for the gather estimator with its path vertices checkpointed,
    replayed, or checkpointed within a 48 GB budget (the chunks that do
    not fit replayed).
    Per mode: iterations/s over --steps timed iterations after --warmup
    (the first iteration sizes the vertex store) and the device memory the
    renderer and its frame hold afterwards.  One JSON line."""
    import torch

    from differentiablepointrendering_b200.build import build_library
    from differentiablepointrendering_b200.device import DeviceFrame
    from differentiablepointrendering_b200.pale import Renderer
    from differentiablepointrendering_b200.scene import jitter_target, make_box_scene, make_surfels

    build_library()
    dev = torch.device("cuda:0")
    w = dict(WORKLOADS["box1m-32view"], spp=args.c3b_passes, adjoint_spp=args.c3b_passes)
    base = dict(settings_for(w), gradients="all")
    pts = make_surfels(w["n"], 1234)
    scene = make_box_scene(w["n"], cameras=w["cams"], resolution=w["res"], points=pts)
    tr = Renderer.from_scene(scene.with_points(jitter_target(pts, 5678)), base)
    tf = DeviceFrame(tr, device=dev)
    tf.forward()
    target = tf.ldr[:, :3].clone()
    torch.cuda.synchronize()
    del tf
    tr.close()
    torch.cuda.empty_cache()
    stream = torch.cuda.current_stream(dev)
    rows = []
    for label, extra in C3B_MODES:
        torch.cuda.synchronize()
        free0, total = torch.cuda.mem_get_info()
        r = Renderer.from_scene(scene, dict(base, **extra))
        frame = DeviceFrame(r, device=dev)
        for _ in range(max(1, args.warmup)):
            frame.forward_loss(target)
            frame.backward()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3 * args.steps)]
        for k in range(args.steps):
            ev[3 * k].record(stream)
            frame.forward_loss(target)
            ev[3 * k + 1].record(stream)
            frame.backward()
            ev[3 * k + 2].record(stream)
        torch.cuda.synchronize()
        fwd = sum(ev[3 * k].elapsed_time(ev[3 * k + 1]) for k in range(args.steps)) / args.steps
        bwd = sum(ev[3 * k + 1].elapsed_time(ev[3 * k + 2]) for k in range(args.steps)) / args.steps
        st = r.stats()
        free1, _ = torch.cuda.mem_get_info()
        grads = {k: float(v.double().norm()) for k, v in frame.grads.items() if k in ("opacity", "albedo")}
        rows.append({"mode": label, "iters_per_s": round(1e3 / (fwd + bwd), 4), "forward_ms": round(fwd, 1),
                     "backward_ms": round(bwd, 1), "device_bytes": int(free0 - free1),
                     "vertex_bytes": int(st["vertex_bytes"]),
                     "chunks_stored": int(st["vertex_chunks_stored"]),
                     "chunks_replayed": int(st["vertex_chunks_replayed"]),
                     "gather_segments": int(st["gather_segments"]), "grad_norms": grads})
        del frame
        r.close()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    print(json.dumps({"metric": "C3b iters/s and device memory, checkpointed vs replayed path vertices",
                      "impl": "ours", "n_gpus": 1, "workload": dict(w, workload="box1m-32view"),
                      "gradients": "all", "steps": args.steps, "warmup": max(1, args.warmup),
                      "device_total_bytes": int(total), "modes": rows}), flush=True)


# ---------------------------------------------------------------- serving
SERVING_SURFELS = tuple(int(round(10000 * 100 ** (k / 7))) for k in range(8))   # 10k .. 1M, log-uniform
SERVING_RES = (128, 256, 512, 1024)
SERVING_SPP = (1, 2, 4, 8, 16, 32, 64)
SERVING_SETTINGS = {"photons": 1000000, "bounces": 8, "forward_passes": 1, "gather_passes": 64,
                    "adjoint_bounces": 8, "adjoint_passes": 64, "gather_radius": 0.01}


def serving_request(rng, names, kind=None, res=None, spp=None):
    """One request of the serving mix: a scene of the eight, a camera of
    resolution uniform in 128..1024 (squared), passes log-uniform in 1..64,
    adjoint depth uniform in 4..8; 70% forward, 30% gradient."""
    from differentiablepointrendering_b200.serving import Request

    s = names[int(rng.integers(len(names)))]
    k = int(rng.integers(len(SERVING_RES))) if res is None else SERVING_RES.index(res)
    cam = int(rng.integers(2)) * len(SERVING_RES) + k
    kind = kind or ("gradient" if rng.uniform() < 0.3 else "forward")
    reso = SERVING_RES[k]
    tgt = rng.uniform(0, 1, (reso, reso, 3)).astype("float32") if kind == "gradient" else None
    passes = spp or SERVING_SPP[int(rng.integers(len(SERVING_SPP)))]
    return Request(s, cam, kind, tgt, passes, int(rng.integers(4, 9)))


def serve_stream(srv, reqs):
    """Submits (arrival time, request) pairs at their times; the served
    latencies, the span, and the same arrivals on the plain path (each
    request alone, in arrival order, on a virtual clock)."""
    import numpy as np

    from differentiablepointrendering_b200.serving import Request

    t0 = time.perf_counter()
    for at, q in reqs:
        delay = t0 + at - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        srv.submit(q)
    for _, q in reqs:
        q.done.wait(900)
        if q.error:
            raise RuntimeError(q.error)
    span = max(q.t_done for _, q in reqs) - t0
    served = np.array([q.latency_ms for _, q in reqs])
    clock, plain, service = 0.0, [], []
    for at, q in reqs:
        p = srv.serve_one(Request(q.scene, q.camera, q.kind, q.target, q.passes, q.depth))
        if p.error:
            raise RuntimeError(p.error)
        clock = max(clock, at) + (p.t_done - p.t_submit)
        plain.append((clock - at) * 1e3)
        service.append((p.t_done - p.t_submit) * 1e3)
    return served, span, np.array(plain), clock, np.array(service)


def plain_light_first(reqs, service_ms, starve_s: float = 5.0):
    """The plain path with the server's light-first order: one request at a
    time, the next one the lightest that has arrived (those waiting longer
    than starve_s first), on a virtual clock of the measured service times;
    returns the latencies (ms) and the end time (s)."""
    import numpy as np

    arr = np.array([at for at, _ in reqs])
    svc = np.asarray(service_ms) / 1e3
    left = set(range(len(reqs)))
    lat = np.zeros(len(reqs))
    clock = 0.0
    while left:
        ready = [i for i in left if arr[i] <= clock]
        if not ready:
            clock = min(arr[i] for i in left)
            continue
        old = [i for i in ready if clock - arr[i] > starve_s]
        i = min(old, key=lambda j: arr[j]) if old else min(ready, key=lambda j: (svc[j], arr[j]))
        clock += svc[i]
        lat[i] = (clock - arr[i]) * 1e3
        left.remove(i)
    return lat, clock


def _pcts(a):
    import numpy as np

    return {"p50_ms": round(float(np.percentile(a, 50)), 2), "p99_ms": round(float(np.percentile(a, 99)), 2)}


def run_serving(args):
    """The serving workload: eight resident box scenes of 10k..1M surfels
    (log-uniform) admitted under a 150 GB HBM budget, and Poisson streams of
    single-view requests (70% forward, 30% gradient; resolution 128..1024
    squared, passes 1..64, depth 4..8) at each rate, served by
    serving.Server in rounds and, for comparison, one request at a time in
    arrival order (the plain path).  Then streams of 512x512 gradient
    requests alone, for their p99 latency.  One JSON line."""
    import numpy as np
    import torch

    from differentiablepointrendering_b200.build import build_library
    from differentiablepointrendering_b200.scene import make_box_scene, make_surfels
    from differentiablepointrendering_b200.serving import Server

    build_library()
    rng = np.random.default_rng(17)
    free, _ = torch.cuda.mem_get_info()
    budget = min(150 * 10 ** 9, int(free * 0.9))
    srv = Server(hbm_budget=budget, max_views=64, max_pixels=1 << 24, max_paths=args.round_paths,
                 settings={"estimator": args.estimator}, policy=args.policy)
    try:
        names = []
        t_admit = time.perf_counter()
        for k, n in enumerate(SERVING_SURFELS):
            name = f"box{n // 1000}k"
            srv.add_scene(name, make_box_scene(n, cameras=2, resolutions=SERVING_RES,
                                               points=make_surfels(n, 1234 + k)), SERVING_SETTINGS)
            names.append(name)
        t_admit = time.perf_counter() - t_admit
        # warm-up: the largest request of each kind twice, so that the
        # executors' wavefront buffers (and the gather estimator's vertex
        # store, sized from the round before) reach their full size before
        # the streams (a buffer that grows inside a stream costs a
        # reallocation in some request's latency)
        for _ in range(2):
            warm = [(0.0, serving_request(rng, names, kind, 1024, SERVING_SPP[-1])) for kind in ("forward", "gradient")]
            serve_stream(srv, warm)
        runs = []
        for rate in args.rates:
            count = max(8, min(args.requests, int(rate * args.seconds)))
            t, reqs = 0.0, []
            for _ in range(count):
                t += rng.exponential(1.0 / rate)
                reqs.append((t, serving_request(rng, names)))
            served, span, plain, clock, service = serve_stream(srv, reqs)
            lf, lf_clock = plain_light_first(reqs, service)
            views = [q.batch_views for _, q in reqs]
            runs.append({"rate_per_s": rate, "requests": count,
                         "served": dict(_pcts(served), requests_per_s=round(count / span, 2),
                                        mean_views_per_round=round(float(np.mean(views)), 2),
                                        max_views_per_round=int(max(views))),
                         "plain": dict(_pcts(plain), requests_per_s=round(count / clock, 2),
                                       service=_pcts(service)),
                         "plain_light_first": dict(_pcts(lf), requests_per_s=round(count / lf_clock, 2))})
        g512 = []
        for spp in (1, 4, 16):
            t, reqs = 0.0, []
            for _ in range(args.requests_512):
                t += rng.exponential(1.0 / args.rate_512)
                reqs.append((t, serving_request(rng, names, "gradient", 512, spp)))
            served, span, plain, clock, service = serve_stream(srv, reqs)
            g512.append({"passes": spp, "rate_per_s": args.rate_512, "requests": len(reqs),
                         "served": _pcts(served), "plain": _pcts(plain), "service_alone": _pcts(service)})
        admitted = srv.admitted_bytes
    finally:
        srv.close()
    print(json.dumps({"metric": "serving latency p50/p99 (ms) and requests/s", "impl": "ours", "n_gpus": 1,
                      "scenes": [{"name": m, "surfels": n} for m, n in zip(names, SERVING_SURFELS)],
                      "scene_settings": SERVING_SETTINGS, "resolutions": SERVING_RES, "passes": SERVING_SPP,
                      "depths": [4, 8], "round_paths": args.round_paths, "estimator": args.estimator,
                      "policy": args.policy,
                      "mix": "70% forward (LDR image of one view), 30% gradient (L2 loss + adjoint of one view)",
                      "budget_bytes": budget, "admitted_bytes": admitted, "admit_s": round(t_admit, 2),
                      "runs": runs, "gradient_512": g512}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--workload", default="box200k", choices=sorted(WORKLOADS))
    ap.add_argument("--skip-cpu", dest="skip_cpu", action="store_true")
    ap.add_argument("--gradients", default="opacity", choices=("opacity", "all"),
                    help="gradient groups of the adjoint: the reference's opacity, or all seven")
    ap.add_argument("--estimator", default="reference", choices=("reference", "gather"),
                    help="backward: the reference's adjoint, or the gather estimator (checkpointed path vertices)")
    ap.add_argument("--skip-extra", dest="skip_extra", action="store_true",
                    help="skip the per-view and request-latency measurements")
    ap.add_argument("--no-tune", dest="no_tune", action="store_true", help="C4 without the autotuner")
    ap.add_argument("--c4", action="store_true", help="only the C4 batched-vs-plain measurement")
    ap.add_argument("--c3b", action="store_true", help="only the C3b checkpoint-vs-replay measurement")
    ap.add_argument("--c3b-passes", dest="c3b_passes", type=int, default=2)
    ap.add_argument("--serving", action="store_true", help="serving benchmark (Poisson request stream)")
    ap.add_argument("--rates", type=float, nargs="*", default=[50.0, 200.0, 500.0, 2000.0])
    ap.add_argument("--seconds", type=float, default=4.0, help="serving: stream length per rate")
    ap.add_argument("--requests", type=int, default=200, help="serving: at most this many requests per rate")
    ap.add_argument("--round-paths", dest="round_paths", type=int, default=1 << 24,
                    help="serving: camera paths (pixels x passes) per round")
    ap.add_argument("--policy", default="light_first", choices=("arrival", "light_first"),
                    help="serving: the order in which a round takes queued requests")
    ap.add_argument("--rate-512", dest="rate_512", type=float, default=20.0)
    ap.add_argument("--requests-512", dest="requests_512", type=int, default=40)
    args = ap.parse_args()
    if args.serving:
        run_serving(args)
        return
    if args.c3b:
        run_c3b(args)
        return
    if args.c4:
        import torch
        from differentiablepointrendering_b200.build import build_library

        build_library()
        dev = torch.device("cuda:0")
        res = c4_measure(dev, tune=not args.no_tune, iterations=max(1, args.steps if args.steps < 5 else 1))
        print(json.dumps({"metric": "C4 iters/s", "value": res["batched_iters_per_s"], "unit": "iters/s",
                          "impl": "ours", "n_gpus": 1, "higher_is_better": True, **res}), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
