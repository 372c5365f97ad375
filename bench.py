#!/usr/bin/env python
"""Benchmark: Mrays/s of the path-tracing hot path on the procedural
2,048,002-triangle icosphere field (400 displaced subdivision-4 icospheres on a
ground quad, Disney materials, 2048x1024 synthetic sky with a 5e4 sun lobe),
1920x1080, 256 spp, max depth 16, Sobol.

One step = one full render of that workload (the reference's
Renderer::renderAll: 64 frames of 4 samples per pixel), issued as one
graph-captured launch of wavefront passes of up to 2^27 path slots (64 spp at
1080p); scene resident in HBM.  Rays = camera + extension + shadow rays traced.

The line also carries the second half of the metric, measured on the
hidden-light room (1024x1024, depth 16): the wall time at which the plain
integrator and the guided, batched one reach relMSE 1e-3 against the FP64
oracle on a 128 x 128 crop (key "convergence"); and the BVH build of the
bench scene by the host SAH builder and by the GPU builder (key "bvh_build").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank renders the full workload with disjoint sample
indices (weak scaling, no data-path collective); value = rays of all ranks /
max-over-ranks time.  --impl reference times the reference's own CPU
implementation (its integrator compiled for the host, oracle/_ref) on the
host cores, on a bounded row sample of the same workload.
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

METRIC = "Mrays/s"
HBM_FALLBACK_GBS = 6650.0


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--spp", type=int, default=256, help="samples per pixel of one step (workload: 256)")
    p.add_argument("--small", action="store_true", help="a small scene for quick checks (not a bench line)")
    p.add_argument("--cpu-sample-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu-baseline", action="store_true",
                   help="skip the CPU baseline leg (profiling runs; the line then carries cpu_baseline null)")
    p.add_argument("--paths-in-flight", type=int, default=0,
                   help="wavefront path slots of the render (0: the autotuner's choice)")
    p.add_argument("--no-autotune", action="store_true",
                   help="render with the library defaults instead of the autotuner's choice")
    p.add_argument("--workload", choices=["render", "batch", "large", "build", "guided"], default="render",
                   help="render: the bench line; batch: the 64-scene uneven batch in one launch; large: the "
                        "20M-triangle 16-camera case; build: host vs GPU BVH build of the bench scene; "
                        "guided: online training then a guided render of the hidden-light room at "
                        "--room-size (a small case for profiling the guide's kernels) (separate lines)")
    p.add_argument("--room-size", type=int, default=512, help="image side of --workload guided")
    p.add_argument("--room-train-spp", type=int, default=4, help="training spp of --workload guided")
    p.add_argument("--guide-infer", choices=["default", "fused", "split_mma", "split_tc", "all"], default="default",
                   help="network evaluation kernels of --workload guided (all: train with the default, then "
                        "time every kind on the same guided render)")
    p.add_argument("--large-spp", type=int, default=512, help="samples per pixel per camera of --workload large")
    p.add_argument("--large-train-spp", type=int, default=64, help="guide training spp of --workload large")
    p.add_argument("--builder", choices=["host", "device"], default="host",
                   help="BVH builder of --workload large: host = the reference's SAH build (node for node), "
                        "device = the GPU builder (linear BVH + treelet restructuring); both build times are "
                        "reported")
    p.add_argument("--no-convergence", action="store_true",
                   help="skip the guided-vs-plain convergence leg (the line then carries convergence null)")
    return p.parse_args()


def workload(small: bool):
    from pathtracingtutorial_b200 import scenes
    if small:
        return scenes.icosphere_field(n_spheres=40, subdiv=3, width=480, height=270, env_size=(512, 256))
    return scenes.icosphere_field()


def config_of(sa, spp):
    return {"workload": f"icosphere_field {sa.meta['triangles']} tri, {int(sa.camera['width'])}x"
                        f"{int(sa.camera['height'])}, {spp} spp, depth {sa.max_depth}, sobol, env 2048x1024",
            "triangles": sa.meta["triangles"], "width": int(sa.camera["width"]), "height": int(sa.camera["height"]),
            "spp": spp, "max_depth": sa.max_depth, "sampler": "sobol", "sample_per_frame": sa.sample_per_frame,
            "l2": "inputs larger than L2 (BVH + triangles ~150 MB > 126 MB L2)"}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", HBM_FALLBACK_GBS)), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def shard_first_frame(rank: int, batches: int) -> int:
    """Rank r renders frames [r * batches, (r + 1) * batches): disjoint sample
    indices (Sobol index = frame * samplePerFrame + i), no data exchange."""
    return rank * batches


def combine_over_ranks(ms: float, rays: float, dist, device: str):
    """Max of the per-rank device times, sum of the rays traced."""
    if dist is None:
        return ms, float(rays)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    r = torch.tensor([float(rays)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(r, op=dist.ReduceOp.SUM)
    return float(t[0]), float(r[0])


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), for the CPU baseline's record."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_arm(args):
    """The reference's own CPU integrator on the host cores, bounded sample."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle.pyoracle import RefHarness
    sa = workload(args.small)
    cfg = config_of(sa, args.spp)
    import numpy as np
    if not RefHarness.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference host build (oracle/_ref) not built"}))
        return
    R = RefHarness()
    cores = os.cpu_count() or 1
    st = np.array([args.spp, sa.sample_per_frame, sa.max_depth, sa.sampler], np.int32)
    h = int(sa.camera["height"])
    # calibrate a row stride so one step is ~cpu_sample_seconds
    _, _, cal = R.render(sa.vertices, sa.faces, sa.materials, sa.camera, st, sa.env, num_frames=1, row0=0,
                         row_step=max(1, h // 8), threads=cores)
    per_row = cal["seconds"] / max(1, len(range(0, h, max(1, h // 8))))
    rows_per_step = max(1, int(args.cpu_sample_seconds / max(per_row, 1e-6)))
    stride = max(1, h // rows_per_step)
    rays = secs = paths = 0.0
    for k in range(args.warmup + args.steps):
        _, _, s = R.render(sa.vertices, sa.faces, sa.materials, sa.camera, st, sa.env, first_frame=k,
                           num_frames=1, row0=k % stride, row_step=stride, threads=cores)
        if k >= args.warmup:
            rays += s["closest_rays"] + s["shadow_rays"]
            secs += s["seconds"]
            paths += s["paths"]
    value = rays / secs / 1e6
    sample = (f"rows y = k mod {stride} (every {stride}th row, {len(range(0, h, stride))} rows x "
              f"{int(sa.camera['width'])} px), 1 frame of {sa.sample_per_frame} spp per step, {int(paths)} paths")
    line = {"metric": METRIC, "value": round(value, 3), "unit": METRIC, "impl": "reference", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(secs / args.steps * 1e3, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": {"value": round(value, 3), "unit": METRIC, "cores": cores, "kind": "reference",
                             "cpu_model": cpu_model(), "build": "reference host sources, g++ -O3",
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def cpu_baseline(sa, spp, seconds):
    """Reference CPU path timed on this host (rank 0, N=1): a bounded sample of
    the workload -- every k-th row, k chosen so one frame takes a fraction of
    `seconds`, then consecutive frames (sample indices as in the full render)
    until `seconds` of CPU time have been spent."""
    import numpy as np
    from oracle.pyoracle import Oracle, RefHarness
    cores = os.cpu_count() or 1
    st = np.array([spp, sa.sample_per_frame, sa.max_depth, sa.sampler], np.int32)
    h = int(sa.camera["height"])
    max_frames = max(1, spp // sa.sample_per_frame)
    rays = secs = paths = 0.0
    frames = 0
    if RefHarness.available():
        R = RefHarness()
        _, _, cal = R.render(sa.vertices, sa.faces, sa.materials, sa.camera, st, sa.env, num_frames=1, row0=0,
                             row_step=max(1, h // 8), threads=cores)
        per_row = cal["seconds"] / len(range(0, h, max(1, h // 8)))
        stride = max(1, int(h / max(1.0, 0.25 * seconds / max(per_row, 1e-6))))
        while secs < seconds and frames < max_frames:
            _, _, s = R.render(sa.vertices, sa.faces, sa.materials, sa.camera, st, sa.env, first_frame=frames,
                               num_frames=1, row0=1, row_step=stride, threads=cores)
            rays += s["closest_rays"] + s["shadow_rays"]
            secs += s["seconds"]
            paths += s["paths"]
            frames += 1
        kind = "reference"
    else:
        O = Oracle()
        prep = O.prepare(sa)
        stride = max(1, h // 16)
        _, s = O.render(prep, sa.sample_per_frame, sa.max_depth, sa.sampler, frames=1, precision=32, rtl=1,
                        row0=1, row_step=stride, threads=cores)
        rays, secs, paths, frames = s["closest_rays"] + s["shadow_rays"], s["seconds"], s["paths"], 1
        kind = "port"
    return {"value": round(float(rays / secs / 1e6), 3), "unit": METRIC, "cores": cores, "kind": kind,
            "cpu_model": cpu_model(),
            "build": "reference host sources, g++ -O3" if kind == "reference" else "oracle restatement, g++ -O2",
            "sample": f"every {stride}th row of {int(sa.camera['width'])}x{h}, {frames * sa.sample_per_frame} spp "
                      f"({frames} frames of {sa.sample_per_frame}), {int(paths)} paths, {int(rays)} rays, "
                      f"{secs:.1f} s"}


ROOM_CROP_FIXTURE = os.path.join(ROOT, "tests", "golden", "room_crop_fp64.npz")
TARGET_RELMSE = 1e-3
GUIDE_SEEDS = (1, 2, 3, 4)   # network initialisations of the convergence leg's guided arm


def crossing_time(trace, target):
    """First checkpoint of a progressive trace [(spp, ms, relmse), ...] whose
    relMSE is at or below `target`, and the time of the crossing
    interpolated log-log between it and the checkpoint before; (None, None)
    when the trace never gets there."""
    import math
    for k, (spp, ms, e) in enumerate(trace):
        if e <= target:
            if k == 0:
                return ms, ms
            s0, m0, e0 = trace[k - 1]
            if e0 <= e or m0 <= 0 or e <= 0:
                return ms, ms
            f = math.log(e0 / target) / math.log(e0 / e)
            return ms, m0 * (ms / m0) ** f
    return None, None


def convergence(local: int, stream, small: bool, plain_cap: int = 8192, guided_cap: int = 4096,
                chunk: int = 64, train_spp: int = 64):
    """Guided + batched vs plain on the hidden-light room (202,002 triangles,
    1024 x 1024, depth 16, Sobol): wall time to relMSE 1e-3 against the FP64
    oracle on the room's central 128 x 128 crop (tests/golden/room_crop_fp64.npz,
    the FP64 restatement at tens of thousands of spp on disjoint sample
    indices; its own noise is recorded with it).

    Plain: the plain integrator (Renderer.render_frames) in chunks of `chunk`
    spp; guided: a guide trained online for `train_spp` spp (timed), then
    rendered through pt_render_batch with the trained guide as the item's
    guide, chunk by chunk (consecutive first frames), the chunks averaged.
    Each arm's clock runs from its start to every checkpoint and includes the
    image read-back (as Renderer::runConvergenceBenchmark, renderer.cu:138-173);
    relMSE = mean over crop pixels and channels of (I - R)^2 / (R^2 + 1e-2).
    The crossing is measured: the first checkpoint at or below 1e-3 (and the
    log-log interpolated crossing between it and the previous checkpoint).
    The guided arm runs once per network seed in GUIDE_SEEDS (the trained
    network depends on its initialisation); its time is the mean of theirs."""
    import numpy as np
    import torch
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    if small or not os.path.exists(ROOM_CROP_FIXTURE):
        return None
    z = np.load(ROOM_CROP_FIXTURE)
    x0, y0, x1, y1 = (int(v) for v in z["crop"])
    ref = z["mean"].astype(np.float64)
    eps = float(z["eps_rel"])
    ref_noise = float(z["noise_relmse"])
    sa = scenes.hidden_light_room(width=int(z["width"]), height=int(z["height"]))
    scene = sa.scene()
    scene.build_accel()
    scene.upload_to_device(local)
    spf = sa.sample_per_frame
    handle = stream.cuda_stream

    def relmse_crop(c):
        return float(np.mean((c - ref) ** 2 / (ref * ref + eps)))

    def relmse(img):
        return relmse_crop(img[y0:y1, x0:x1, :3].astype(np.float64))

    def sync():
        torch.cuda.synchronize(local)

    # plain arm
    r = pt.Renderer(scene, device=local, stream=handle)
    r.reset_accumulation()
    scene.set_frame_count(0)
    r.render_frames(chunk // spf)            # warm-up: graph capture and arena
    sync()
    r.reset_accumulation()
    scene.set_frame_count(0)
    plain = []
    t0 = time.perf_counter()
    spp = 0
    while spp < plain_cap:
        r.render_frames(chunk // spf)
        sync()
        img = r.download_current_image()
        spp += chunk
        e = relmse(img)
        plain.append((spp, (time.perf_counter() - t0) * 1e3, e))
        if e <= TARGET_RELMSE:
            break
    r.integrator.close()
    r.film.close()

    # guided arm, once per network seed: online training, then batched
    # rendering with the trained guide.  The trained network (and so the
    # crossing) depends on the network's initialisation; the arm's time is the
    # mean over the seeds, each seed's crossing is reported.
    def guided_arm(seed):
        g = pt.Guide(scene, seed=seed)
        pt.render_batch([(scene, chunk, 200_000, None, g)], mode=pt.BATCH_WAVEFRONT, autotune=False)   # warm-up
        rg = pt.Renderer(scene, device=local, stream=handle)
        sync()
        t0 = time.perf_counter()
        g.attach(rg.integrator, pt.Guide.TRAIN)
        rg.reset_accumulation()
        scene.set_frame_count(100_000)           # training samples are independent of the image's
        rg.render_frames(train_spp // spf)
        sync()
        train_ms = (time.perf_counter() - t0) * 1e3
        g.attach(rg.integrator, pt.Guide.OFF)
        rg.integrator.close()
        rg.film.close()
        trace = []
        acc = None
        spp = 0
        while spp < guided_cap:
            imgs, _, _ = pt.render_batch([(scene, chunk, spp // spf, None, g)], mode=pt.BATCH_WAVEFRONT,
                                         autotune=False)
            # the whole image is read back; only the scored crop is averaged on the host
            img = imgs[0][y0:y1, x0:x1, :3].astype(np.float64)
            acc = img if acc is None else acc + (img - acc) * (chunk / (spp + chunk))
            spp += chunk
            e = relmse_crop(acc)
            trace.append((spp, (time.perf_counter() - t0) * 1e3, e))
            if e <= TARGET_RELMSE:
                break
        return g, train_ms, trace

    runs = []
    for seed in GUIDE_SEEDS:
        g, train_ms, trace = guided_arm(seed)
        runs.append((seed, train_ms, trace))
        if seed != GUIDE_SEEDS[0]:
            g.close()
        else:
            g_first = g
    g = g_first
    _, train_ms, guided = runs[0]
    # stage breakdown of one chunk of each arm (CUDA events around every launch;
    # separate renders after both clocks stopped)
    breakdown = {}
    rg = pt.Renderer(scene, device=local, stream=handle)
    for arm, mode in (("plain", pt.Guide.OFF), ("guided", pt.Guide.USE)):
        g.attach(rg.integrator, mode)
        scene.update_settings(flags=pt.FLAG_STAGE_TIMING | pt.FLAG_NO_GRAPH)
        rg.integrator.reset_stats()
        rg.reset_accumulation()
        scene.set_frame_count(300_000)
        rg.render_frames(chunk // spf)
        sync()
        st = rg.integrator.stats()
        breakdown[arm] = {k: round(st[k], 2) for k in ("extend_ms", "shade_ms", "shadow_ms", "guide_ms", "other_ms")}
        breakdown[arm]["rays"] = int(st["camera_rays"] + st["extension_rays"] + st["shadow_rays"])
        scene.update_settings(flags=0)
    g.attach(rg.integrator, pt.Guide.OFF)
    rg.integrator.close()
    rg.film.close()
    g.close()
    tp_chk, tp = crossing_time(plain, TARGET_RELMSE)
    per_seed = []
    for seed, tms, tr in runs:
        chk, t = crossing_time(tr, TARGET_RELMSE)
        per_seed.append({"seed": seed, "train_ms": round(tms, 1), "time_to_relmse_1e-3_ms": None if t is None else round(t, 1),
                         "spp": tr[-1][0], "speedup": None if (t is None or tp is None) else round(tp / t, 3)})
    seed_times = [p["time_to_relmse_1e-3_ms"] for p in per_seed]
    tg = None if any(t is None for t in seed_times) else sum(seed_times) / len(seed_times)
    tg_chk = crossing_time(guided, TARGET_RELMSE)[0]
    # secondary: the same with the reference's own noise taken out
    tpc = crossing_time([(a, b, c - ref_noise) for a, b, c in plain], TARGET_RELMSE)[1]
    tgcs = [crossing_time([(a, b, c - ref_noise) for a, b, c in tr], TARGET_RELMSE)[1] for _, _, tr in runs]
    tgc = None if any(t is None for t in tgcs) else sum(tgcs) / len(tgcs)

    def brief(tr):
        keep = {2 ** k for k in range(6, 16)}
        return [[a, round(b, 1), round(c, 6)] for a, b, c in tr if a in keep or (a, b, c) == tr[-1]]

    return {"scene": f"hidden_light_room {len(sa.faces)} tri, {int(z['width'])}x{int(z['height'])}, "
                     f"depth {sa.max_depth}, sobol",
            "reference": f"FP64 oracle, crop x {x0}-{x1} y {y0}-{y1}, {int(z['spp'])} spp, "
                         f"noise relMSE {ref_noise:.2e}",
            "eps_rel": eps, "chunk_spp": chunk,
            "plain": {"path": "Renderer.render_frames (pt_renderer_render_frames)", "trace": brief(plain)},
            "guided": {"path": "pt_render_batch, wavefront item with its trained guide", "train_spp": train_spp,
                       "network_seeds": list(GUIDE_SEEDS), "per_seed": per_seed,
                       "train_ms": round(train_ms, 1), "trace": brief(guided),
                       "note": "time = mean over the network seeds; trace and first checkpoint of the first seed"},
            "time_to_relmse_1e-3_ms": {"plain": None if tp is None else round(tp, 1),
                                       "guided": None if tg is None else round(tg, 1)},
            "first_checkpoint_below_1e-3_ms": {"plain": None if tp_chk is None else round(tp_chk, 1),
                                               "guided": None if tg_chk is None else round(tg_chk, 1)},
            "noise_corrected_time_ms": {"plain": None if tpc is None else round(tpc, 1),
                                        "guided": None if tgc is None else round(tgc, 1)},
            "guided_speedup": None if (tp is None or tg is None) else round(tp / tg, 3),
            "target_speedup": 3.0,
            "stage_ms_per_chunk": breakdown}


def build_leg(sa):
    """BVH build of the bench scene: the reference-order host SAH build once,
    the GPU builder (default options) after one warm-up, median of three."""
    import statistics
    host = sa.scene()
    t0 = time.perf_counter()
    host.build_accel()
    host_ms = (time.perf_counter() - t0) * 1e3
    del host
    dev = sa.scene()
    dev.build_accel(builder="device")
    runs = [dev.build_accel(builder="device") for _ in range(3)]
    total = statistics.median(r["total_ms"] for r in runs)
    return {"host_ms": round(host_ms, 1), "device_ms": round(total, 1),
            "device_kernels_ms": round(statistics.median(r["device_ms"] for r in runs), 2),
            "speedup": round(host_ms / total, 2), "note": "bench.py --workload build adds the trace rate of each tree"}


def ours(args):
    import numpy as np
    import torch
    import pathtracingtutorial_b200 as pt

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    sa = workload(args.small)
    spp = args.spp
    scene = sa.scene()
    scene.build_accel()
    scene.upload_to_device(local)
    # the library's autotuner picks the traversal shape and queue capacity
    # (untimed; cached per device and scene class), unless fixed by the caller
    tuned = None
    if args.paths_in_flight > 0:
        scene.update_settings(paths_in_flight=args.paths_in_flight)
    elif not args.no_autotune:
        tuned = scene.autotune()
    spf = sa.sample_per_frame
    batches = (spp + spf - 1) // spf
    stream = torch.cuda.Stream(device=local)
    handle = stream.cuda_stream
    renderer = pt.Renderer(scene, device=local, stream=handle)
    frame0 = shard_first_frame(rank, batches)   # disjoint sample indices per rank

    def step():
        # Renderer::renderAll over `batches` frames: one graph-captured launch
        renderer.reset_accumulation()
        scene.set_frame_count(frame0)
        renderer.render_frames(batches)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        renderer.integrator.reset_stats()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clocks:
            barrier()
            ev0.record(stream)
            for _ in range(args.steps):
                step()
            ev1.record(stream)
            barrier()
        ms = ev0.elapsed_time(ev1)
    st = renderer.integrator.stats()
    rays = st["camera_rays"] + st["extension_rays"] + st["shadow_rays"]
    # whole-job: rays of all ranks over the slowest rank's time
    ms, total_rays = combine_over_ranks(ms, rays, dist, f"cuda:{local}")
    value = total_rays / (ms / 1e3) / 1e6

    # e2e through the public API: host->device scene upload, render, image read back
    cam = scene.camera
    img = np.zeros((int(cam["height"]), int(cam["width"]), 4), np.float32)
    e2e_ms = []
    e2e_rays = 0
    for k in range(max(1, min(args.steps, 3)) + 1):
        barrier()
        t0 = time.perf_counter()
        scene.upload_to_device(local)
        out, sts = pt.render(scene, spp, stats=True)
        barrier()
        if k > 0:
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
            e2e_rays = sts["camera_rays"] + sts["extension_rays"] + sts["shadow_rays"]
    info = scene.info()
    e2e_val = e2e_rays / (statistics.median(e2e_ms) / 1e3) / 1e6 * world

    # instrumented replicas of one step: (1) per-stage CUDA events on the
    # kernels as timed; (2) traversal counters (node pops and triangle tests of
    # the reference's tree walk: same rays, same visit order)
    def replica(flags):
        scene.update_settings(flags=flags)
        renderer.integrator.reset_stats()
        with torch.cuda.stream(stream):
            step()
        torch.cuda.synchronize()
        return renderer.integrator.stats()
    ist = replica(pt.FLAG_STAGE_TIMING)
    cst = replica(pt.FLAG_COUNT_TRAVERSAL)
    scene.update_settings(flags=0)
    closest = cst["camera_rays"] + cst["extension_rays"]
    pops = closest + 2 * cst["node_visits"]
    alg_bytes = 32.0 * pops + 36.0 * cst["triangle_tests"]
    launches = max(1, ist["extend_launches"])
    per_launch_ms = ist["extend_ms"] / launches
    achieved = alg_bytes / launches / (per_launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = units = None
    tp = os.path.join(ROOT, "profiles", "extend_traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            prof = json.load(f)
        traffic = prof.get("dram_bytes_per_launch")
        u = prof.get("units_small_case")
        if u:   # the L2 / L1 / issue fractions beside the HBM one (ncu, small case)
            units = {k: u[k] for k in ("l2_throughput_of_peak", "l1tex_throughput_of_peak", "dram_throughput_of_peak",
                                       "issue_active_of_peak", "lanes_per_warp_instruction")}
            units["source"] = "profiles/extend_traffic.json (ncu --set full, 4-spp case)"
    stage_total = ist["extend_ms"] + ist["shade_ms"] + ist["shadow_ms"] + ist["other_ms"]

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    # release this render's wavefront state (tens of GB) before the next legs
    renderer.integrator.close()
    renderer.film.close()
    del renderer
    conv = None
    if world == 1 and not args.no_convergence:
        with torch.cuda.stream(stream):
            conv = convergence(local, stream, args.small)
    cpu = cpu_baseline(sa, spp, args.cpu_sample_seconds) if world == 1 and not args.no_cpu_baseline else None
    build = build_leg(sa) if world == 1 else None
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(config_of(sa, spp), launch={
            "paths_in_flight": scene.settings().paths_in_flight, "trace_block": scene.settings().trace_block,
            "stack_depth": scene.settings().stack_depth,
            "autotune": None if tuned is None else {k: tuned[k] for k in ("calib_spp", "best_ms", "default_ms",
                                                                         "candidates")}}),
        "rays_per_step": total_rays / args.steps / world,
        "ray_classes": {"camera": st["camera_rays"] // args.steps, "extension": st["extension_rays"] // args.steps,
                        "shadow": st["shadow_rays"] // args.steps},
        "e2e": {"value": round(e2e_val, 2), "unit": METRIC, "ms_per_step": round(statistics.median(e2e_ms), 2),
                "h2d_bytes_per_step": int(info["device_bytes"]), "d2h_bytes_per_step": int(img.nbytes),
                "path": "pt_scene_upload + pt_render (host arrays -> device, 256 spp, image -> host)"},
        "roofline": {"kernel": "k_extend (closest-hit traversal)", "bound": "hbm", "achieved": round(achieved, 1),
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic, "units": units, "algorithmic_bytes_per_launch": alg_bytes / launches,
                     "avg_launch_ms": round(per_launch_ms, 4), "launches": launches,
                     "stage_ms": {"extend": round(ist["extend_ms"], 2), "shade": round(ist["shade_ms"], 2),
                                  "shadow": round(ist["shadow_ms"], 2), "other": round(ist["other_ms"], 2)},
                     "extend_share": round(ist["extend_ms"] / max(stage_total, 1e-9), 3),
                     "note": "achieved = (32 B x node pops + 36 B x triangle tests of the reference's "
                             "traversal of the same rays) / extend launch time, CUDA events on a stage-timed "
                             "replica of one step; traffic = ncu dram read+write per launch (profiles/)"},
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
        "gpu_launches": int(st["kernel_launches"]),
        "convergence": conv,
        "bvh_build": build,
    }
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def batch_workload(args):
    """--workload batch: the uneven batch (64 scenes like the icosphere field,
    triangles log-uniform in 1k..2M, resolutions from {256^2, 512^2, 1024^2,
    1280x720}, 16..512 spp, depth 12, one shared sky) rendered by one
    pt.render_batch call (the autotuner picks persistent or wavefront mode on
    a first call), against rendering the 64 scenes one after another with
    pt.render.  Wall time of each call (it returns host images), rays counted
    by the kernels."""
    import torch
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    torch.cuda.set_device(0)
    batch = scenes.uneven_batch(n_scenes=64)
    ss = []
    for sa in batch:
        sc = sa.scene()
        sc.build_accel()
        sc.upload_to_device(0)
        ss.append(sc)
    items = [(sc, sa.spp) for sc, sa in zip(ss, batch)]
    _, _, cfg = pt.render_batch(items, autotune=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, st, _ = pt.render_batch(items, block_size=cfg["block_size"], blocks_per_sm=cfg["blocks_per_sm"],
                               chunk_spp=cfg["chunk_spp"], autotune=False, mode=cfg["mode"],
                               paths_in_flight=cfg["paths_in_flight"])
    t_batch = time.perf_counter() - t0
    rays = st["camera_rays"] + st["extension_rays"] + st["shadow_rays"]
    t0 = time.perf_counter()
    rays_seq = 0
    for sc, sa in zip(ss, batch):
        _, s1 = pt.render(sc, sa.spp, stats=True)
        rays_seq += s1["camera_rays"] + s1["extension_rays"] + s1["shadow_rays"]
    t_seq = time.perf_counter() - t0
    mode = {pt.BATCH_PERSISTENT: "persistent", pt.BATCH_WAVEFRONT: "wavefront"}.get(cfg["mode"], str(cfg["mode"]))
    print(json.dumps({
        "metric": METRIC, "workload": "uneven batch: 64 scenes, %d triangles, %d pixels x spp, depth 12"
        % (sum(len(sa.faces) for sa in batch), st["paths"]),
        "value": round(rays / t_batch / 1e6, 2), "unit": METRIC, "seconds": round(t_batch, 3),
        "paths": int(st["paths"]), "rays": int(rays),
        "sequential": {"value": round(rays_seq / t_seq / 1e6, 2), "seconds": round(t_seq, 3)},
        "batch_speedup": round(t_seq / t_batch, 3),
        "autotuned": {"mode": mode, "block_size": cfg["block_size"], "blocks_per_sm": cfg["blocks_per_sm"],
                      "chunk_spp": cfg["chunk_spp"], "paths_in_flight": cfg["paths_in_flight"],
                      "tuned_ms": round(cfg["tuned_ms"], 2)}}))


def large_workload(args):
    """--workload large: the combined large case -- about 20M triangles
    (displaced icospheres and tetrahedral clutter, flattened), Disney
    materials, the synthetic sky and 32 small area lights, 16 cameras at
    1920x1080, depth 16 -- rendered as ONE batch of 16 camera items of the one
    uploaded scene, plain and guided (the guide trained online on the first
    camera first).  --large-spp samples per pixel per camera (the full case,
    the default, is 512).  Camera 0's image of each arm is judged on a 128 x
    128 crop against the FP64 oracle's (tests/golden/large_crop_fp64.npz, when
    present): relMSE as measured, and with the oracle's own recorded noise
    taken out."""
    import numpy as np
    import torch
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    sa, cams = scenes.large_scene()
    t_gen = time.perf_counter() - t0
    scene = sa.scene()
    t0 = time.perf_counter()
    scene.build_accel()
    t_build = time.perf_counter() - t0
    d = sa.scene()
    d.build_accel(builder="device")                            # warm-up: first CUDA use, allocator
    dev_build = d.build_accel(builder="device")
    if args.builder == "device":
        scene = d
    del d
    t0 = time.perf_counter()
    scene.upload_to_device(0)
    t_upload = time.perf_counter() - t0
    info = scene.info()
    spp = args.large_spp
    items = [(scene, spp, 0, c) for c in cams]
    pt.render_batch([(scene, 4, 0, c) for c in cams[:2]], mode=pt.BATCH_WAVEFRONT)   # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    imgs_plain, st, cfg = pt.render_batch(items, mode=pt.BATCH_WAVEFRONT)
    t_plain = time.perf_counter() - t0
    rays = st["camera_rays"] + st["extension_rays"] + st["shadow_rays"]
    g = pt.Guide(scene, seed=1)
    r = pt.Renderer(scene)
    g.attach(r.integrator, pt.Guide.TRAIN)
    r.reset_accumulation()
    scene.set_frame_count(100_000)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r.render_frames(max(1, args.large_train_spp // sa.sample_per_frame))
    r.synchronize()
    t_train = time.perf_counter() - t0
    t0 = time.perf_counter()
    imgs_guided, stg, _ = pt.render_batch([(scene, spp, 0, c, g) for c in cams])
    t_guided = time.perf_counter() - t0
    rays_g = stg["camera_rays"] + stg["extension_rays"] + stg["shadow_rays"]
    g.close()
    crop_eval = None
    fx = os.path.join(ROOT, "tests", "golden", "large_crop_fp64.npz")
    if os.path.exists(fx):
        z = np.load(fx)
        x0, y0, x1, y1 = (int(v) for v in z["crop"])
        ref = z["mean"].astype(np.float64)
        eps, noise = float(z["eps_rel"]), float(z["noise_relmse"])

        def relmse(img):
            c = img[y0:y1, x0:x1, :3].astype(np.float64)
            return float(np.mean((c - ref) ** 2 / (ref * ref + eps)))
        ep, eg = relmse(imgs_plain[0]), relmse(imgs_guided[0])
        crop_eval = {"reference": f"FP64 oracle, camera 0, crop x {x0}-{x1} y {y0}-{y1}, {int(z['spp'])} spp",
                     "reference_noise_relmse": round(noise, 6),
                     "plain_relmse": round(ep, 6), "guided_relmse": round(eg, 6),
                     "plain_relmse_noise_corrected": round(ep - noise, 6),
                     "guided_relmse_noise_corrected": round(eg - noise, 6)}
    print(json.dumps({
        "metric": METRIC, "workload": f"large scene {info['num_faces']} tri ({args.builder}-built BVH "
                                      f"{info['num_bvh_nodes']} nodes, depth {info['bvh_max_depth']}), 16 cameras "
                                      f"1920x1080, {spp} spp each, depth 16",
        "builder": args.builder,
        "host_seconds": {"generate": round(t_gen, 1), "bvh_build": round(t_build, 1), "upload": round(t_upload, 2)},
        "device_build": {k: (round(v, 2) if isinstance(v, float) else v) for k, v in dev_build.items()},
        "device_bytes": int(info["device_bytes"]),
        "plain": {"value": round(rays / t_plain / 1e6, 2), "unit": METRIC, "seconds": round(t_plain, 3),
                  "paths": int(st["paths"]), "rays": int(rays)},
        "guided": {"value": round(rays_g / t_guided / 1e6, 2), "unit": METRIC, "seconds": round(t_guided, 3),
                   "train_spp": args.large_train_spp, "train_seconds": round(t_train, 3), "rays": int(rays_g)},
        "crop_relmse": crop_eval}))


def build_workload(args):
    """--workload build: the bench scene (2,048,002 triangles) built by the
    reference-order host SAH builder and by the GPU builder (defaults: linear
    BVH, three treelet passes), each tree then traced by the same integrator:
    64 spp of the 1080p render, best of two, CUDA events.  --steps timed GPU
    builds after --warmup untimed ones (their median is reported)."""
    import statistics
    import torch
    import pathtracingtutorial_b200 as pt
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    sa = workload(args.small)

    def trace_rate(scene):
        r = pt.Renderer(scene, stream=stream.cuda_stream)
        best = None
        for _ in range(3):
            r.reset_accumulation()
            scene.set_frame_count(0)
            r.integrator.reset_stats()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            r.render_frames(64 // sa.sample_per_frame)
            e1.record(stream)
            torch.cuda.synchronize()
            st = r.integrator.stats()
            rate = (st["camera_rays"] + st["extension_rays"] + st["shadow_rays"]) / e0.elapsed_time(e1) / 1e3
            best = rate if best is None else max(best, rate)
        return best

    host = sa.scene()
    t0 = time.perf_counter()
    host.build_accel()
    host_s = time.perf_counter() - t0
    host.upload_to_device(0)
    hi = host.info()
    host_rate = trace_rate(host)
    del host
    dev = sa.scene()
    for _ in range(max(1, args.warmup)):
        dev.build_accel(builder="device")
    runs = [dev.build_accel(builder="device") for _ in range(max(1, args.steps))]
    dev.upload_to_device(0)
    di = dev.info()
    dev_rate = trace_rate(dev)
    med = {k: round(statistics.median(r[k] for r in runs), 2) for k in runs[0] if k.endswith("_ms")}
    print(json.dumps({
        "metric": "BVH build ms", "workload": f"{sa.name} {di['num_faces']} tri", "steps": len(runs),
        "host": {"build_ms": round(host_s * 1e3, 1), "nodes": hi["num_bvh_nodes"], "depth": hi["bvh_max_depth"],
                 "trace_mrays": round(host_rate, 1)},
        "device": {"build_ms": med, "nodes": di["num_bvh_nodes"], "depth": di["bvh_max_depth"],
                   "trace_mrays": round(dev_rate, 1)},
        "build_speedup": round(host_s * 1e3 / med["total_ms"], 2),
        "trace_ratio": round(dev_rate / host_rate, 3)}))


GUIDE_INFER = {"default": 0, "fused": 1, "split_mma": 2, "split_tc": 3}


def guided_workload(args):
    """Online training for --room-train-spp, then --spp guided samples per
    pixel of the hidden-light room at --room-size squared; stage times of the
    guided render.  A profiling case for the guide's kernels.  With
    --guide-infer all, the trained guide then renders the same --spp samples
    once per inference kind with per-stage CUDA events (the network's stage
    time of each kind, and the image mean)."""
    import torch
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    sa = scenes.hidden_light_room(width=args.room_size, height=args.room_size)
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    kinds = list(GUIDE_INFER)[1:] if args.guide_infer == "all" else [args.guide_infer]
    g = pt.Guide(s, seed=1, inference=GUIDE_INFER[kinds[0]])
    t0 = time.perf_counter()
    img, g, st = pt.render_guided(s, train_spp=args.room_train_spp, spp=args.spp, guide=g)
    secs = time.perf_counter() - t0
    info = g.info()
    per_kind = {}
    if len(kinds) > 1:
        r = pt.Renderer(s, device=0)
        g.attach(r.integrator, pt.Guide.USE)
        s.update_settings(flags=pt.FLAG_STAGE_TIMING | pt.FLAG_NO_GRAPH)
        spf = sa.sample_per_frame
        for kind in kinds * 2:   # the second round is the one kept (the first warms up)
            g.set_inference(GUIDE_INFER[kind])
            r.integrator.reset_stats()
            r.reset_accumulation()
            s.set_frame_count(0)
            r.render_frames((args.spp + spf - 1) // spf)
            torch.cuda.synchronize()
            k = r.integrator.stats()
            per_kind[kind] = {"guide_ms": round(k["guide_ms"], 2), "extend_ms": round(k["extend_ms"], 2),
                              "shade_ms": round(k["shade_ms"], 2), "shadow_ms": round(k["shadow_ms"], 2),
                              "mean": round(float(r.download_current_image()[..., :3].mean()), 6)}
        s.update_settings(flags=0)
        g.attach(r.integrator, pt.Guide.OFF)
        r.integrator.close()
        r.film.close()
    g.close()
    print(json.dumps({
        "metric": "guided render", "workload": f"{sa.name} {len(sa.faces)} tri, {args.room_size}^2, "
                                              f"depth {sa.max_depth}",
        "train_spp": args.room_train_spp, "spp": args.spp, "seconds": round(secs, 3),
        "inference": kinds[0], "optimiser_steps": info["steps"], "mean": float(img[..., :3].mean()),
        "rays": int(st["camera_rays"] + st["extension_rays"] + st["shadow_rays"]),
        "kernel_launches": int(st["kernel_launches"]), "per_inference_kind": per_kind or None}))


def main():
    args = parse_args()
    if args.workload == "guided":
        guided_workload(args)
    elif args.workload == "build":
        build_workload(args)
    elif args.workload == "batch":
        batch_workload(args)
    elif args.workload == "large":
        large_workload(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
