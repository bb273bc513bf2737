"""Throughput benchmark of the snow/water substep (particle-substeps/s) on B200.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Workload: the scene at the scale of the reference's published figures (5,888 water +
147,928 snow particles, 52,016 boundary particles, seeded synthetic lattice), one step = one frame = 4 substeps of dt = 1/240 s
with 3 solver iterations.  `value` is timed on the device with CUDA events around each
frame (state resident in HBM, L2 flushed between frames); `e2e` goes through the C-ABI
call with the per-frame host I/O of the reference (positions, velocities and temperatures
of the live particles of both sets copied from pinned host memory before the frame and
back after it, the buffers the reference maps from GL each frame).  Multi-GPU runs are independent replicas
(one scene per rank, no collective in the step); `value` is the sum over ranks divided by
the slowest rank's time.

The line also carries "batched": 64 scenes of uneven size (log-uniform 2k-40k particles)
stepped as one batch, against the same scenes stepped one after another through the
plain entry point (--no-batched skips it; on N ranks the 64 scenes are split between the
ranks, each stepping its share as one batch with no exchange inside a step, and the block
reports all scenes' particle-substeps over the slowest rank's time); "adjoint": a
differentiable rollout of config 3 to frame 60 (240 substeps, forward with checkpoints
every 10 + backward) against the same substeps run plain (--no-adjoint skips it); "large":
3 frames of the 1.18M-particle config 4 in a widened domain (--no-large skips it);
"long_window": every frame 0-99 of the scene from rest (--long-frames); "fp64_error": the
first 24 frames against the FP64 oracle with the heat-energy drift of both runs
(--fp64-frames, --no-fp64).

--precision-study runs the config-4 precision study instead (FP64 oracle comparison of the
first frames, GPU heat-energy drift over 600 frames, per-kernel HBM fractions).

--impl reference times the CPU restatement of the same substep (FP32, all host threads) on
the same frames of the same scene (W warm-up frames, K timed frames of 4 substeps), the
only CPU implementation of this path: the reference itself runs it only on a GPU.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-substeps/s @154k particles (config 1)"
UNIT = "particle-substeps/s"
SUBSTEPS = 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scene", default="config1")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--fp64-frames", type=int, default=24)
    ap.add_argument("--long-frames", type=int, default=100)
    ap.add_argument("--precision-study", action="store_true")
    ap.add_argument("--precision-fp64-frames", type=int, default=10)
    ap.add_argument("--precision-energy-frames", type=int, default=600)
    ap.add_argument("--precision-quirks", default="fixed", choices=["fixed", "reference"])
    ap.add_argument("--profile-out", default="")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def slowest(values_ms, ws, dev):
    """Per-rank device times -> their maximum over the ranks (one all_reduce for the list)."""
    if ws == 1:
        return [float(v) for v in values_ms]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values_ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def job_rate(units_per_rank, ws, ms):
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return ws * units_per_rank / (ms / 1000.0)


# ----------------------------------------------------------------- clocks sampling
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                       "-lms", "50", "-i", str(dev)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        # nvidia-smi takes a moment to start: wait (at most 2 s) for its first row, so that
        # the timed region that follows is sampled from its start
        t0 = time.perf_counter()
        while self.p is not None and time.perf_counter() - t0 < 2.0:
            if os.path.getsize(self.f.name) > 0 or self.p.poll() is not None:
                break
            time.sleep(0.01)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ----------------------------------------------------------------- CPU baseline
def cpu_baseline(scene_name, max_seconds=25.0, max_substeps=None):
    """FP32 oracle (project CPU restatement) on the same scene, all host threads."""
    from snowsimulation_b200 import scene
    from oracle.oracle import OracleWorld
    w = getattr(scene, scene_name)()
    cores = os.cpu_count() or 1
    o = OracleWorld(w, 32, threads=cores).setup()
    n = w.n_sph + w.n_dem
    done, t0 = 0, time.perf_counter()
    while True:
        o.step()
        done += 1
        el = time.perf_counter() - t0
        if el > max_seconds * 0.5 or (max_substeps and done >= max_substeps):
            break
    return {"value": n * done / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d substep(s) of %s (%d particles), FP32 C oracle, OpenMP %d threads, %.1f s"
                      % (done, scene_name, n, cores, el)}


def reference_cpu_baselines(water_pos, snow_pos, links, snow_mass, h, dt, iters=3, max_seconds=4.0):
    """The reference's own CPU code near this path, timed on the host (reported baselines;
    neither routine is the substep): NeighborSearch::SpatialSearch over the water set, and
    ConstraintSolver::SolveXPBDConstraints over one distance constraint per interlink of the
    scene at rest, `iters` iterations (the interlink stage of one substep)."""
    from oracle import cpu_ref
    if not cpu_ref.available():
        return {"unavailable": "oracle/_ref/libsnowcpuref.so not built (needs the reference sources)"}
    out = {}
    nw = len(water_pos)
    _, t1 = cpu_ref.spatial_search(water_pos, h, calls=1)
    calls = int(max(1, min(500, max_seconds / max(t1, 1e-6))))
    pairs, sec = cpu_ref.spatial_search(water_pos, h, calls=calls)
    out["spatial_search"] = {
        "value": nw / sec, "unit": "particles searched/s", "cores": cpu_ref.SPATIAL_SEARCH_THREADS,
        "kind": "reference",
        "sample": "NeighborSearch::SpatialSearch (NeighborSearch.cpp:154-259) on the %d water particles, "
                  "radius %.3f m, its fixed 1 m hash grid; %d calls, %.3f ms per call, %d neighbour pairs"
                  % (nw, h, calls, sec * 1e3, pairs)}
    a, b, rest = links
    _, t1 = cpu_ref.xpbd_links(snow_pos, a, b, rest, snow_mass, dt, iters=iters, calls=1)
    calls = int(max(1, min(20, max_seconds / max(t1, 1e-6))))
    _, sec = cpu_ref.xpbd_links(snow_pos, a, b, rest, snow_mass, dt, iters=iters, calls=calls)
    out["xpbd_links"] = {
        "value": len(a) * iters / sec, "unit": "constraint projections/s", "cores": cpu_ref.XPBD_THREADS,
        "kind": "reference",
        "sample": "ConstraintSolver::SolveXPBDConstraints (ConstraintSolver.cpp:51-72) over %d DistanceConstraints "
                  "(the scene's interlinks at rest) on %d snow particles, %d iterations; %d solves, %.1f ms per solve"
                  % (len(a), len(snow_pos), iters, calls, sec * 1e3)}
    return out


# ----------------------------------------------------------------- error vs FP64
def fp64_error(scene_name, dev, frames=24):
    """The GPU run of the timed scene against the FP64 oracle from the same start, frame by
    frame (particles matched by track id, whichever set holds them): maximum position,
    velocity and temperature differences, and the total heat energy sum(m C T) and momentum
    sum(m v) of both runs (FP64 reductions: snowb_energy_momentum on the GPU state, the
    oracle's own sums on its state), with their drift from the start."""
    import numpy as np
    from snowsimulation_b200 import scene
    from snowsimulation_b200.world import Simulation
    from oracle.oracle import OracleWorld
    w = getattr(scene, scene_name)()
    sim = Simulation(w, device=dev).setup()
    o = OracleWorld(w, 64, threads=os.cpu_count() or 1).setup()
    out = []

    def by_id(world_sets):
        ids, xs, vs, ts = [], [], [], []
        for d, n in world_sets:
            ids.append(d["trackId"][:n]); xs.append(d["positions"][:n]); vs.append(d["velocity"][:n])
            ts.append(d["T"][:n])
        ids = np.concatenate(ids)
        order = np.argsort(ids)
        f64 = lambda a: np.concatenate(a)[order].astype(np.float64)
        return ids[order], f64(xs), f64(vs), f64(ts)

    e0g, e0o = sim.energy_momentum(), o.energy_momentum()
    t0 = time.perf_counter()
    for f in range(frames):
        sim.step(substeps=SUBSTEPS)
        for _ in range(SUBSTEPS):
            o.step()
        H = sim.to_host()
        ig, xg, vg, tg = by_id(((H.sph, H.n_sph), (H.dem, H.n_dem)))
        io, xo, vo, to = by_id(((o.w.sph, o.w.n_sph), (o.w.dem, o.w.n_dem)))
        same = np.array_equal(ig, io)
        eg, eo = sim.energy_momentum(), o.energy_momentum()
        rec = {"frame": f, "same_particles": bool(same), "sizes": [H.n_sph, H.n_dem],
               "sizes_fp64": [o.w.n_sph, o.w.n_dem]}
        if same:
            rec["pos_max_m"] = float(np.abs(xg - xo).max())
            rec["vel_max_mps"] = float(np.abs(vg - vo).max())
            rec["T_max_C"] = float(np.abs(tg - to).max())
        rec["energy_J"] = eg[0]
        rec["energy_fp64_J"] = eo[0]
        rec["energy_drift_rel"] = (eg[0] - e0g[0]) / abs(e0g[0])
        rec["energy_drift_fp64_rel"] = (eo[0] - e0o[0]) / abs(e0o[0])
        rec["momentum"] = eg[1:]
        rec["momentum_fp64"] = eo[1:]
        out.append(rec)
    el = time.perf_counter() - t0
    fin = [r for r in out if r.get("same_particles")]
    summary = {}
    if fin:
        summary = {"pos_max_m": max(r["pos_max_m"] for r in fin), "vel_max_mps": max(r["vel_max_mps"] for r in fin),
                   "T_max_C": max(r["T_max_C"] for r in fin),
                   "energy_rel_diff_max": max(abs(r["energy_J"] - r["energy_fp64_J"]) / abs(r["energy_fp64_J"])
                                              for r in out),
                   "first_contact_frame": next((r["frame"] for r in fin if r["T_max_C"] > 0.0), None)}
    return {"workload": "%s from rest, %d frames of %d substeps" % (scene_name, frames, SUBSTEPS),
            "oracle": "FP64 C restatement of the substep (oracle/), reference quirks, OpenMP %d threads, %.0f s"
                      % (os.cpu_count() or 1, el),
            "summary": summary, "per_frame": out}


# ----------------------------------------------------------------- reference arm
def run_reference(args):
    """The CPU restatement of the substep on the same workload as the other arm: the same
    scene from rest, W untimed frames, then K timed frames of SUBSTEPS substeps (wall
    clock), all host threads; rank 0 only."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from snowsimulation_b200 import scene
    from oracle.oracle import OracleWorld
    w = getattr(scene, args.scene)()
    cores = os.cpu_count() or 1
    o = OracleWorld(w, 32, threads=cores).setup()
    n = w.n_sph + w.n_dem
    warm = max(3, args.warmup)
    for _ in range(warm * SUBSTEPS):
        o.step()
    budget = 240.0   # bound on the timed region (a slow host times fewer frames and says so)
    t0 = time.perf_counter()
    done = 0
    while done < args.steps:
        for _ in range(SUBSTEPS):
            o.step()
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    val = n * SUBSTEPS * done / el
    workload = workload_name(args.scene, w)
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": done, "warmup": warm, "ms_per_step": 1000.0 * el / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload, "substeps_per_step": SUBSTEPS, "iterations": w.iterations,
                       "quirks": "reference", "parallelism": "single", "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": "frames %d-%d (%d substeps each) of %s from rest, FP32 C restatement of the "
                                       "substep (oracle/), OpenMP %d threads; the reference runs this path only on "
                                       "a GPU" % (warm, warm + done - 1, SUBSTEPS, args.scene, cores)},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    gpu = reference_gpu_runner(args.scene, args.warmup, min(args.steps, 20))
    if gpu is not None:
        line["gpu_runner"] = gpu
    print(json.dumps(line))
    return 0


def workload_name(scene_name, w):
    return ("%s: %d water + %d snow + %d boundary particles, 1 step = 1 frame = %d substeps (dt 1/240 s, "
            "%d iterations), seeded lattice" % (scene_name, w.n_sph, w.n_dem, w.n_b, SUBSTEPS, w.iterations))


def reference_gpu_runner(scene_name, warmup, frames):
    """The reference's own CUDA substep (cuda_simulation.cu compiled unmodified with the
    project's fast math, oracle/_ref/libsnowref.so) on this GPU over the same scene, for
    comparison with the other arm: frames of 4 substeps timed with CUDA events on the
    default stream, which the reference uses (each of its calls synchronises)."""
    try:
        import torch
        from oracle import ref_runner
    except ImportError:
        return None
    if not torch.cuda.is_available():
        return None
    if not ref_runner.available("fast"):
        return {"unavailable": "oracle/_ref/libsnowref.so not built (needs the reference sources)"}
    from snowsimulation_b200 import scene
    w = getattr(scene, scene_name)()
    n = w.n_sph + w.n_dem
    r = ref_runner.RefWorld(w, "fast").setup()
    try:
        for _ in range(max(3, warmup) * SUBSTEPS):
            r.step()
        torch.cuda.synchronize()
        ms = []
        for _ in range(frames):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(SUBSTEPS):
                r.step()
            b.record()
            b.synchronize()
            ms.append(a.elapsed_time(b))
    finally:
        r.close()
    per = sum(ms) / len(ms)
    return {"value": n * SUBSTEPS / (per / 1000.0), "unit": UNIT, "ms_per_step": per, "frames": len(ms),
            "warmup_frames": max(3, warmup),
            "workload": "%s, 1 step = 1 frame = %d substeps, the same frames as the other arm" % (scene_name, SUBSTEPS),
            "build": "the reference's cuda_simulation.cu + cuda_tool.cu, unmodified, fast math, sm_100a"}


# ----------------------------------------------------------------- batched vs plain
def batched_compare(frames, dev, flush, ws=1, rank=0):
    """The 64 scenes of config 2 (uneven sizes, log-uniform 2k-40k particles) stepped as one
    batch, and the same scenes stepped one after another through the plain entry point (each
    with its own cached substep graph).  Both in the fixed-quirks mode, in which the batch
    equals the independent runs bit for bit.  Device time with CUDA events per frame.  On
    several ranks the scenes are split between them (batch.shard_scenes), each rank steps
    its own share with no exchange inside a step, and combine_batched() joins the per-rank
    figures after the timed region."""
    import torch
    from snowsimulation_b200 import scene
    from snowsimulation_b200.abi import QUIRKS_FIXED
    from snowsimulation_b200.batch import BatchSimulation, shard_scenes
    from snowsimulation_b200.world import Simulation

    every = scene.config2(seed=0)
    sizes = [w.n_sph + w.n_dem for w in every]
    mine = shard_scenes(sizes, ws, rank)
    worlds = [every[i] for i in mine]
    part = {"frames": frames, "scenes_total": len(every), "particles_total": sum(sizes),
            "boundary_total": sum(w.n_b for w in every), "scenes": mine,
            "particle_substeps": sum(sizes[i] for i in mine) * SUBSTEPS * frames,
            "batch_ms": 0.0, "plain_ms": 0.0, "water_after": [], "snow_after": []}
    if not worlds:   # fewer scenes than ranks
        return part
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        ms = []
        for _ in range(frames):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(a.elapsed_time(b))
        return sum(ms)

    plain = [Simulation(w, device=dev, quirks=QUIRKS_FIXED).setup() for w in worlds]

    def plain_frame():
        for sim in plain:
            sim.step(substeps=SUBSTEPS, sync=False, use_graph=True)

    for _ in range(3):
        plain_frame()
    torch.cuda.synchronize(dev)
    part["plain_ms"] = timed(plain_frame)
    del plain
    torch.cuda.empty_cache()

    batch = BatchSimulation(worlds, device=dev).setup()

    def batch_frame():
        batch.step(substeps=SUBSTEPS, sync=False, use_graph=True)

    for _ in range(3):
        batch_frame()
    torch.cuda.synchronize(dev)
    part["batch_ms"] = timed(batch_frame)
    batch.read_sizes()
    part["water_after"], part["snow_after"] = batch.scene_counts()
    del batch
    torch.cuda.empty_cache()
    return part


def combine_batched(parts):
    """The batched block of the bench line from every rank's share (rank order): all ranks'
    particle-substeps over the slowest rank's device time, for the batch and for the plain
    scene-by-scene runs, and each scene's live particles after the timed frames."""
    p0 = parts[0]
    n_sc, frames = p0["scenes_total"], p0["frames"]
    owner = {}
    for r, p in enumerate(parts):
        for i in p["scenes"]:
            if i in owner:
                raise RuntimeError("scene %d stepped by ranks %d and %d" % (i, owner[i], r))
            owner[i] = r
    if sorted(owner) != list(range(n_sc)):
        raise RuntimeError("scenes not stepped by any rank: %s" % sorted(set(range(n_sc)) - set(owner)))
    ps = sum(p["particle_substeps"] for p in parts)
    b_ms = max(p["batch_ms"] for p in parts)
    p_ms = max(p["plain_ms"] for p in parts)
    water, snow = [0] * n_sc, [0] * n_sc
    for p in parts:
        for k, i in enumerate(p["scenes"]):
            water[i], snow[i] = p["water_after"][k], p["snow_after"][k]
    return {"workload": "config2: %d scenes, %d water+snow particles (log-uniform 2k-40k per scene) + %d boundary, "
                        "1 step = 1 frame = %d substeps, fixed quirks" % (n_sc, p0["particles_total"],
                                                                          p0["boundary_total"], SUBSTEPS),
            "frames": frames, "value": ps / (b_ms / 1000.0), "unit": UNIT, "ms_per_step": b_ms / frames,
            "plain_value": ps / (p_ms / 1000.0), "plain_ms_per_step": p_ms / frames,
            "speedup_vs_plain": p_ms / b_ms,
            "parallelism": "scenes split over %d ranks" % len(parts) if len(parts) > 1 else "single",
            "scenes_per_rank": [len(p["scenes"]) for p in parts],
            "particles_per_rank": [p["particle_substeps"] // (SUBSTEPS * frames) for p in parts],
            "particles_after": {"water": sum(water), "snow": sum(snow)}}


# ----------------------------------------------------------------- large scene
def large_scene(frames, dev, seed, flush, warmup=2):
    """Config 4 (1,048,576 snow + 131,072 water, walls at +-1.5 m, 128^3 grid): device time of
    `frames` graph-replayed frames of 4 substeps after `warmup` frames, reference quirks."""
    import torch
    from snowsimulation_b200 import scene
    from snowsimulation_b200.world import Simulation
    w = scene.config4(seed=seed)
    sim = Simulation(w, device=dev).setup()
    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        sim.step(substeps=SUBSTEPS, sync=False, use_graph=True)
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(frames):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.step(substeps=SUBSTEPS, sync=False, use_graph=True)
        b.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(a.elapsed_time(b))
    sim.read_sizes()
    n = w.n_sph + w.n_dem
    res = {"workload": "config4: %d water + %d snow + %d boundary, 128^3 grid, walls +-1.5 m, frames %d-%d"
                       % (w.n_sph, w.n_dem, w.n_b, warmup, warmup + frames - 1),
           "frames": frames, "ms_per_step": sum(ms) / frames,
           "value": n * SUBSTEPS * frames / (sum(ms) / 1000.0), "unit": UNIT,
           "sizes_after": [sim.n_sph, sim.n_dem]}
    del sim
    torch.cuda.empty_cache()
    return res


# ----------------------------------------------------------------- long window
def long_window(frames, dev, seed, flush, scene_name="config1"):
    """Device time of every frame 0..frames-1 of the scene from rest (graph replay, L2
    flushed before each frame outside the events): the mean over the whole window and per
    20-frame span, where the cost changes as the water melts into the snow."""
    import torch
    from snowsimulation_b200 import scene
    from snowsimulation_b200.world import Simulation
    w = getattr(scene, scene_name)(seed=seed)
    sim = Simulation(w, device=dev).setup()
    stream = torch.cuda.current_stream(dev)
    ms = []
    for _ in range(frames):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.step(substeps=SUBSTEPS, sync=False, use_graph=True)
        b.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(a.elapsed_time(b))
    sim.read_sizes()
    n = w.n_sph + w.n_dem
    spans = {"%d-%d" % (k, min(k + 19, frames - 1)): sum(ms[k:k + 20]) / len(ms[k:k + 20]) for k in range(0, frames, 20)}
    res = {"workload": "%s from rest, frames 0-%d, 1 frame = %d substeps" % (scene_name, frames - 1, SUBSTEPS),
           "ms_per_frame_mean": sum(ms) / frames, "value": n * SUBSTEPS * frames / (sum(ms) / 1000.0),
           "unit": UNIT, "ms_per_frame_by_span": spans, "sizes_after": [sim.n_sph, sim.n_dem],
           "note": "the frame-0 graph capture happens before the first timed event"}
    del sim
    torch.cuda.empty_cache()
    return res


# ----------------------------------------------------------------- precision study (config 4)
def precision_study(dev, fp64_frames=10, energy_frames=600, profile_frames=2, quirks="fixed"):
    """The large scene (1,048,576 snow + 131,072 water, 128^3 grid, walls at +-1.5 m) from
    rest: (1) the FP32 GPU run against the FP64 oracle run of the same scene, frame by frame
    for `fp64_frames` frames (particles matched by track id): position, velocity and
    temperature errors and both runs' heat energy; (2) the GPU run continued to
    `energy_frames` frames with its FP64 heat-energy and momentum reductions every 10
    frames (drift from the start); (3) the per-kernel device time over `profile_frames`
    frames (CUDA-event nodes in the substep graph) against the algorithmic bytes of each
    kernel: achieved GB/s and fraction of the measured HBM peak, taken right after (1).
    quirks: "fixed" (the intended physics) or "reference".  With the reference's quirks the
    heat pass sums each particle's own cell 27 times (Q7), which with conductivities of
    600 and 2500 W/mK puts the explicit snow-snow conduction step above its stability limit
    once the melt brings temperature gradients into the snow, so a long run blows up."""
    import numpy as np
    import torch
    from snowsimulation_b200 import scene, bytes_model, _native
    from snowsimulation_b200.world import Simulation
    from oracle.oracle import OracleWorld
    from snowsimulation_b200.abi import QUIRKS_FIXED, QUIRKS_REFERENCE
    qm = QUIRKS_FIXED if quirks == "fixed" else QUIRKS_REFERENCE
    w = scene.config4(seed=0)
    sim = Simulation(w, device=dev, quirks=qm).setup()
    t0 = time.perf_counter()
    o = OracleWorld(w, 64, qm, threads=os.cpu_count() or 1).setup()

    def by_id(sets):
        ids = np.concatenate([d["trackId"][:n] for d, n in sets])
        order = np.argsort(ids)
        cat = lambda f: np.concatenate([d[f][:n] for d, n in sets])[order].astype(np.float64)
        return ids[order], cat("positions"), cat("velocity"), cat("T")

    e0g, e0o = sim.energy_momentum(), o.energy_momentum()
    rows = []
    for f in range(fp64_frames):
        sim.step(substeps=SUBSTEPS)
        for _ in range(SUBSTEPS):
            o.step()
        H = sim.to_host()
        ig, xg, vg, tg = by_id(((H.sph, H.n_sph), (H.dem, H.n_dem)))
        io, xo, vo, to = by_id(((o.w.sph, o.w.n_sph), (o.w.dem, o.w.n_dem)))
        eg, eo = sim.energy_momentum(), o.energy_momentum()
        r = {"frame": f, "sizes": [H.n_sph, H.n_dem], "sizes_fp64": [o.w.n_sph, o.w.n_dem],
             "energy_drift_rel": (eg[0] - e0g[0]) / abs(e0g[0]), "energy_drift_fp64_rel": (eo[0] - e0o[0]) / abs(e0o[0])}
        if np.array_equal(ig, io):
            r.update(pos_max_m=float(np.abs(xg - xo).max()), vel_max_mps=float(np.abs(vg - vo).max()),
                     T_max_C=float(np.abs(tg - to).max()))
        rows.append(r)
        print("precision frame %d: %s" % (f, json.dumps(r)), file=sys.stderr, flush=True)
    t_fp64 = time.perf_counter() - t0
    del o
    # per-kernel table over the next frames
    lib = sim.lib
    for _ in range(2):   # the graphs of these frames, captured before the profiled ones
        sim.step(substeps=SUBSTEPS, sync=False, use_graph=True)
    lib.snowb_profile_begin()
    for _ in range(profile_frames):
        sim.step(substeps=SUBSTEPS, sync=False, use_graph=True)
    buf = C.create_string_buffer(1 << 16)
    _native.check(lib.snowb_profile_end(buf, len(buf)))
    sim.read_sizes()
    peak, peak_kind = peaks()
    table = []
    for line in buf.value.decode().splitlines():
        nm, c, t = line.split()
        c, t = int(c), float(t)
        base = nm.split("<")[0]
        kb = bytes_model.kernel_bytes(base, sim.n_sph, sim.n_dem, sim.n_b)
        if kb is not None and base == "k_density" and "true" in nm:
            kb += bytes_model.PASS["L"] * (sim.n_sph + sim.n_dem + sim.n_b)
        row = {"kernel": nm, "launches_per_frame": c / profile_frames, "ms_per_frame": t / profile_frames}
        if kb is not None:
            gbs = kb * c / (t / 1000.0) / 1e9
            row.update(algorithmic_bytes_per_launch=kb, achieved_GBs=gbs, hbm_frac=gbs / peak)
        table.append(row)
    table.sort(key=lambda r: -r["ms_per_frame"])
    prof_at = fp64_frames + 2
    drift = []
    for f in range(fp64_frames + 2 + profile_frames, energy_frames):
        sim.step(substeps=SUBSTEPS, sync=False, use_graph=True)
        if (f + 1) % 10 == 0 or f == energy_frames - 1:
            sim.read_sizes()
            e = sim.energy_momentum()
            drift.append({"frame": f, "energy_drift_rel": (e[0] - e0g[0]) / abs(e0g[0]), "momentum": e[1:],
                          "sizes": [sim.n_sph, sim.n_dem]})
    return {"workload": "config4: %d water + %d snow + %d boundary, 128^3 grid, walls +-1.5 m, from rest, %s quirks"
                        % (w.n_sph, w.n_dem, w.n_b, quirks),
            "fp64": {"frames": fp64_frames, "oracle": "FP64 C restatement, OpenMP %d threads, %.0f s"
                                                      % (os.cpu_count() or 1, t_fp64), "per_frame": rows},
            "energy": {"frames": energy_frames, "start_J": e0g[0], "every_10_frames": drift},
            "kernels": {"frames": "%d-%d" % (prof_at, prof_at + profile_frames - 1), "peak_GBs": peak,
                        "peak_kind": peak_kind, "table": table}}


# ----------------------------------------------------------------- adjoint vs plain
def adjoint_compare(substeps, dev, seed, checkpoint_every=10):
    """Config 3 (1,024 water on 8,192 snow with interlinks, phase change off): device time of
    `substeps` plain substeps (graph replay) against a differentiable rollout of the same
    substeps (forward with checkpoints + backward: recomputation with the tape on and the
    reverse kernels), loss = snow-position MSE + temperature MSE, gradients w.r.t. the
    water's initial velocities and k_refreezing, k_stretch, k_water, k_snow."""
    import torch
    from snowsimulation_b200 import scene
    from snowsimulation_b200.abi import QUIRKS_FIXED
    from snowsimulation_b200.adjoint import loss_fn, params_of, restore, rollout, snapshot
    from snowsimulation_b200.world import Simulation

    w = scene.config3(seed=seed)
    sim = Simulation(w, device=dev, quirks=QUIRKS_FIXED).setup()
    n = sim.n_sph + sim.n_dem
    start = snapshot(sim)
    stream = torch.cuda.current_stream(dev)

    def ev_time(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record(stream)
        out = fn()
        b.record(stream)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b), out

    for _ in range(2):   # warm-up (graph capture)
        restore(sim, start)
        sim.step(substeps=substeps, use_graph=True)
    restore(sim, start)
    plain_ms, _ = ev_time(lambda: sim.step(substeps=substeps, use_graph=True))
    restore(sim, start)
    theta = params_of(sim)
    v0 = sim.sph.t["velocity"][:sim.n_sph].clone()
    with torch.no_grad():
        _, xd, _, Td = rollout(sim, v0, theta, substeps, checkpoint_every)
    tx, tT = xd + 0.005, Td + 1.0

    def adj():
        restore(sim, start)
        vv = v0.clone().requires_grad_(True)
        th = theta.clone().requires_grad_(True)
        _, xd, _, Td = rollout(sim, vv, th, substeps, checkpoint_every)
        L = loss_fn(xd, Td, tx, tT, 1e-4)
        L.backward()
        return th.grad

    adj()   # warm-up (tape and reverse buffers)
    adj_ms, g = ev_time(adj)
    return {"workload": "config3: %d water + %d snow + %d boundary, %d substeps, checkpoint every %d, fixed quirks"
                        % (sim.n_sph, sim.n_dem, sim.n_b, substeps, checkpoint_every),
            "plain_ms_per_substep": plain_ms / substeps, "adjoint_ms_per_substep": adj_ms / substeps,
            "adjoint_over_plain": adj_ms / plain_ms,
            "plain_value": n * substeps / (plain_ms / 1000.0), "adjoint_value": n * substeps / (adj_ms / 1000.0),
            "unit": UNIT, "grad_params": [float(x) for x in g]}


# ----------------------------------------------------------------- our arm
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.precision_study:
        import torch
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        print(json.dumps(precision_study(dev, args.precision_fp64_frames, args.precision_energy_frames,
                                         quirks=args.precision_quirks)))
        return 0
    import torch
    import torch.distributed as dist
    from snowsimulation_b200 import scene, bytes_model, _native
    from snowsimulation_b200.world import Simulation

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    w = getattr(scene, args.scene)(seed=rank)
    sim = Simulation(w, device=dev).setup()
    lib = sim.lib
    n_part = w.n_sph + w.n_dem
    rest_state = None
    if ws == 1 and not args.no_cpu_baseline:
        from oracle import cpu_ref
        H0 = sim.to_host()
        rest_state = (H0.sph["positions"][: H0.n_sph].copy(), H0.dem["positions"][: H0.n_dem].copy(),
                      cpu_ref.link_pairs(H0.dem["connect_record"], H0.dem["connect_length"], H0.n_dem, H0.maxc),
                      float(H0.dem["mass"][0]))
        del H0
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2

    def frame(sync=False):
        sim.step(substeps=SUBSTEPS, sync=sync, use_graph=True)

    for _ in range(max(3, args.warmup)):
        frame()
    torch.cuda.synchronize(dev)

    # ---- device-timed frames (inputs resident; L2 flushed between frames, outside the events)
    clocks = Clocks(local)
    cnt0 = C.c_uint64(0)
    lib.snowb_launch_count(C.byref(cnt0))
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record(stream)
        frame()
        evs[k][1].record(stream)
    torch.cuda.synchronize(dev)
    cnt1 = C.c_uint64(0)
    lib.snowb_launch_count(C.byref(cnt1))
    clk = clocks.stop()
    ms = [a.elapsed_time(b) for a, b in evs]
    tot_ms = sum(ms)
    ms_sorted = sorted(ms)
    pct = {"ms_p10": ms_sorted[int(0.1 * (len(ms) - 1))], "ms_p50": statistics.median(ms),
           "ms_p90": ms_sorted[int(round(0.9 * (len(ms) - 1)))]}
    sim.read_sizes()
    tot_ms = slowest([tot_ms], ws, dev)[0]
    value = job_rate(n_part * SUBSTEPS * args.steps, ws, tot_ms)
    ms_per_step = tot_ms / args.steps

    # ---- end to end through the C-ABI call with host buffers, over the same frames of the
    # scene as the timed region: a second, identical simulation warmed up the same way (the
    # scene's cost changes as the water melts into the snow, so later frames would not compare)
    del sim
    sim = Simulation(getattr(scene, args.scene)(seed=rank), device=dev).setup()
    for _ in range(max(3, args.warmup)):
        frame()
    torch.cuda.synchronize(dev)
    fields = ("positions", "velocity", "T")
    host = {(s, f): torch.empty_like(getattr(sim, s).t[f], device="cpu").pin_memory()
            for s in ("sph", "dem") for f in fields}
    for (s, f), hb in host.items():
        hb.copy_(getattr(sim, s).t[f])
    sim.read_sizes()

    def live(s):   # particles of the set (the slots beyond are padding)
        return sim.n_sph if s == "sph" else sim.n_dem

    e_ms, h2d_tot, d2h_tot = [], 0, 0
    if ws > 1:
        dist.barrier()
    for k in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for (s, f), hb in host.items():   # this step's inputs: the live particles of each set
            n = live(s)
            getattr(sim, s).t[f][:n].copy_(hb[:n], non_blocking=True)
            h2d_tot += hb[:n].numel() * hb.element_size()
        frame(sync=True)                       # the reference contract: sizes back on the host
        for (s, f), hb in host.items():   # its results, for the sizes after the step
            n = live(s)
            hb[:n].copy_(getattr(sim, s).t[f][:n], non_blocking=True)
            d2h_tot += hb[:n].numel() * hb.element_size()
        b.record(stream)
        b.synchronize()
        e_ms.append(a.elapsed_time(b))
    h2d = h2d_tot // args.steps
    d2h = d2h_tot // args.steps
    e_tot = sum(e_ms)
    e_tot = slowest([e_tot], ws, dev)[0]
    e2e = job_rate(n_part * SUBSTEPS * args.steps, ws, e_tot)

    # ---- per-kernel device time over the same frames as the timed region: a second,
    # identical simulation is warmed up the same way, then its substep graph is captured
    # with a CUDA event node around every kernel and replayed for the timed frames
    del sim
    sim = Simulation(getattr(scene, args.scene)(seed=rank), device=dev).setup()
    for _ in range(max(3, args.warmup)):
        frame()
    torch.cuda.synchronize(dev)
    prof_frames = min(args.steps, 4)
    lib.snowb_profile_begin()
    for _ in range(prof_frames):
        frame()
    buf = C.create_string_buffer(1 << 16)
    _native.check(lib.snowb_profile_end(buf, len(buf)))
    prof = {}
    for line in buf.value.decode().splitlines():
        nm, c, t = line.split()
        prof[nm] = (int(c), float(t))
    if args.profile_out and rank == 0:
        with open(args.profile_out, "w") as f:
            tot = sum(t for _, t in prof.values())
            for nm, (c, t) in sorted(prof.items(), key=lambda x: -x[1][1]):
                f.write("%-22s launches %5d  total %9.3f ms  share %5.1f%%\n" % (nm, c, t, 100 * t / tot))
    def base(nm):
        return nm.split("<")[0]
    modeled = {nm: v for nm, v in prof.items()
               if bytes_model.kernel_bytes(base(nm), sim.n_sph, sim.n_dem, sim.n_b) is not None}
    top = max(modeled, key=lambda nm: modeled[nm][1])
    c, t = modeled[top]
    c_frames = prof_frames
    per_launch_s = t / c / 1000.0
    kb = bytes_model.kernel_bytes(base(top), sim.n_sph, sim.n_dem, sim.n_b)
    if base(top) == "k_density" and "true" in top:     # density + lambda in one pass
        kb += bytes_model.PASS["L"] * (sim.n_sph + sim.n_dem + sim.n_b)
    traffic = None
    winst = None
    tfile = os.path.join(ROOT, "profiles", "dram_traffic_config1.txt")
    if os.path.exists(tfile):   # per-launch DRAM bytes (and warp instructions) from an ncu capture
        for line in open(tfile):
            parts = line.split()
            if len(parts) >= 2 and parts[0] == top:
                traffic = float(parts[1])
                if len(parts) >= 3:
                    winst = float(parts[2])
    peak, peak_kind = peaks()
    achieved = kb / per_launch_s / 1e9
    # The dominant kernel issues instructions (IEEE divisions and square roots of the
    # bit-exact arithmetic) far more than it moves bytes: its warp instructions per launch
    # (ncu) over the live launch time, against the issue peak of 4 schedulers per SM at the
    # sampled SM clock.
    issue = None
    if winst:
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
        peak_issue = sms * 4 * mhz * 1e6 / 1e9
        issue = {"kernel": top, "warp_instructions_per_launch": winst, "source": "ncu (profiles/)",
                 "achieved": winst / per_launch_s / 1e9, "peak": peak_issue, "unit": "G warp-instructions/s",
                 "frac": winst / per_launch_s / 1e9 / peak_issue,
                 "peak_basis": "%d SMs x 4 schedulers x %.0f MHz (sampled)" % (sms, mhz)}
    sub_bytes = bytes_model.substep_bytes(sim.n_sph, sim.n_dem, sim.n_b, w.iterations)
    sub_gbs = sub_bytes * SUBSTEPS / (ms_per_step / 1000.0) / 1e9

    del sim
    batched_res = None
    if not args.no_batched:
        part = batched_compare(min(args.steps, 5), dev, flush, ws, rank)
        parts = [part]
        if ws > 1:   # after the timed frames: every rank's share to every rank
            parts = [None] * ws
            dist.all_gather_object(parts, part)
        batched_res = combine_batched(parts)

    large_res = None
    if not args.no_large:
        large_res = large_scene(3, dev, rank, flush)
        if ws > 1:
            ms_max = slowest([large_res["ms_per_step"]], ws, dev)[0]
            n = large_res["value"] * large_res["ms_per_step"] / 1000.0
            large_res["value"] = job_rate(n, ws, ms_max)
            large_res["ms_per_step"] = ms_max
    long_res = long_window(args.long_frames, dev, rank, flush, args.scene) if args.long_frames > 0 else None
    if long_res is not None and ws > 1:
        ms_max = slowest([long_res["ms_per_frame_mean"]], ws, dev)[0]
        long_res["value"] = job_rate(long_res["value"] * long_res["ms_per_frame_mean"] / 1000.0, ws, ms_max)
        long_res["ms_per_frame_mean"] = ms_max
    adjoint_res = None
    if not args.no_adjoint:
        adjoint_res = adjoint_compare(240, dev, rank)

    if rank != 0:
        if ws > 1:
            dist.destroy_process_group()
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_per_step, "frame_ms_percentiles": pct,
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(args.scene, w),
                   "substeps_per_step": SUBSTEPS, "iterations": w.iterations,
                   "quirks": "reference", "parallelism": "replicas" if ws > 1 else "single",
                   "l2": "flushed between timed steps (256 MB write)"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e_tot / args.steps},
        "gpu_launches": int(cnt1.value - cnt0.value),
        "clocks": clk,
        "roofline": {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": kb, "avg_launch_ms": per_launch_s * 1000.0,
                     "launches_per_step": c / c_frames},
        "issue_roofline": issue,
        "substep_roofline": {"algorithmic_bytes": sub_bytes, "achieved_GBs": sub_gbs,
                             "frac": sub_gbs / peak},
        "kernel_ms_per_step": {nm: t / prof_frames for nm, (c, t) in sorted(prof.items(), key=lambda x: -x[1][1])},
    }
    if not args.no_batched:
        line["batched"] = batched_res
    if adjoint_res is not None:
        line["adjoint"] = adjoint_res
    if large_res is not None:
        line["large"] = large_res
    if long_res is not None:
        line["long_window"] = long_res
    if ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.scene)
        line["cpu_baseline"]["reference_cpu"] = reference_cpu_baselines(
            rest_state[0], rest_state[1], rest_state[2], rest_state[3], h=float(w.params.effective_radius),
            dt=1.0 / (60.0 * SUBSTEPS))
    if ws == 1 and not args.no_fp64:
        line["fp64_error"] = fp64_error(args.scene, dev, args.fp64_frames)
    print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
