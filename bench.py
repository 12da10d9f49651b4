"""Throughput benchmark of the Radiance path (one JSON line on stdout).

Workload: the 1024x768, 256 spp render of a 1.31M-triangle displaced
icosphere (subdivision 8, 4-octave value-noise displacement of amplitude 0.15)
inside the Cornell-style box, 20 patch materials (50 % Lambert albedo
U[0.2,0.9]^3, 50 % Beckmann roughness U[0.05,0.8]), one ceiling light,
max depth 8 (maxBounce 7), seeded synthetic data.  One step = one full
render of that image = 201,326,592 camera paths.  The estimator is the
reference's (the same arithmetic the reference arm times).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value      Msamples/s of the whole job, device-timed with CUDA events on the
           render stream, max over ranks; inputs resident in HBM.
e2e        Msamples/s through the public C ABI from host arrays: scene upload,
           GPU BVH build, render and the film's device-to-host copy each step.
roofline   the closest-hit traversal kernel (k_extend): algorithmic bytes per
           launch (nodes x 80 B + triangles x 48 B + rays x 48 B, counted by
           the counting build on the same workload) / its mean launch time.
cpu_baseline / --impl reference
           the reference's own CPUMulticoreTracer::execute compiled from its
           sources (oracle/_ref/cr_ref), on this host's cores, on a bounded
           sample of the same workload (full resolution, fewer spp).
batch      the batched workload (64 scenes of uneven size, resolution and spp)
           as one batch replayed from a CUDA graph, against one call per
           scene; the closest-hit L2 roofline over the batch's scenes and the
           reference on a window of every 8th scene; rank 0 at N = 1 only.
guiding    time to relMSE 1e-3, plain MIS vs learned guiding (tensor-core
           inference and online training included), on the occluded-light
           scene at 1024x1024 (see guided_vs_plain); the guide inference
           kernel's tensor and L2 rooflines and the reference on a 1-spp
           render of the scene; rank 0 at N = 1 only.
config0    the small box scene at its full configuration (256x256, 64 spp,
           depth 8), the one workload both arms run identically: device and
           end-to-end rates, the L2 roofline, the reference on the same
           render; rank 0 at N = 1 only.
config4    the large combined run (21M triangles, 3840x2160, depth 12): plain
           and guided rates, HBM roofline, window time to relMSE 1e-3 and the
           reference on that window; rank 0 at N = 1 only.
Multi-GPU: one process per GPU; each rank renders the workload with its own
seed (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "oracle"))  # the CPU-baseline leg only

WIDTH, HEIGHT, SPP, LEVEL, MAX_BOUNCE = 1024, 768, 256, 8, 7
METRIC = ("Msamples/s (camera paths per second), plain wavefront, 1024x768x256spp, 1.31M-tri displaced icosphere; "
          "time-to-relMSE 1e-3 guided vs plain in 'guiding'")
NODE_BYTES, TRI_BYTES, RAY_BYTES = 80, 48, 32 + 16
# the guide's MLP: 5 layers of 64 x 64 (2 FLOP per multiply-add) per inferred
# path, and 48 hash-grid gathers (12 levels x 4 cell edges) to encode it
GUIDE_FLOPS_PER_ROW, GUIDE_GATHERS_PER_ROW = 2 * 64 * 64 * 5, 48
C0_WORKLOAD = ("config0: box scene (20 triangles, 2 spheres, ceiling light), 256x256 at 64 spp, depth 8, "
               "reference estimator")


def load_pkg():
    """The package directory `cuda-raytracer_b200`, imported as cuda_raytracer_b200."""
    import importlib.util
    if "cuda_raytracer_b200" in sys.modules:
        return sys.modules["cuda_raytracer_b200"]
    pkg = os.path.join(ROOT, "cuda-raytracer_b200")
    spec = importlib.util.spec_from_file_location("cuda_raytracer_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cuda_raytracer_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def replica_seed(rank, k):
    """Seed of timed step k on `rank`: every replica renders independent samples."""
    return 7 + 1000 * rank + k


def job_throughput(ms_local, samples_local, device, world):
    """Whole-job Msamples/s of the replicas: all ranks' samples over the slowest
    rank's device time (ms); returns (value, ms_max, samples_all)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms_local, float(samples_local)], dtype=torch.float64, device=device)
    if world > 1:
        mx = t[:1].clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = t[1:].clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        t = torch.cat([mx, sm])
    ms_max, samples_all = float(t[0].item()), float(t[1].item())
    return samples_all / (ms_max / 1e3) / 1e6, ms_max, int(samples_all)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def measured_bf16():
    """Dense BF16 tensor-core peak (burst, TFLOP/s) measured on this GPU type
    (MEASURED_PEAKS.json), else an earlier measurement of the same part."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def profiled_traffic(name="k_extend_traffic.json"):
    """DRAM bytes per unit (ray or row) of a kernel from a committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return None


def make_workload(tmpdir):
    load_pkg()
    from cuda_raytracer_b200 import scenes
    desc = scenes.config1(level=LEVEL, width=WIDTH, height=HEIGHT, spp=SPP)
    path = scenes.write_scene(desc, tmpdir)
    return desc, path


# ---------------------------------------------------------------------------- reference arm
def reference_rate(scene_json, steps, warmup, spp, width=WIDTH, height=HEIGHT):
    """Reference CPU Radiance path (oracle/_ref/cr_ref bench) on all host threads."""
    import oracle
    threads = os.cpu_count() or 1
    r = subprocess.run([oracle.REF_BIN, "bench", os.path.basename(scene_json), str(width), str(height), str(spp),
                        str(threads), str(MAX_BOUNCE), str(steps + warmup)], cwd=os.path.dirname(scene_json),
                       capture_output=True, text=True, timeout=3600, check=True)
    runs = [json.loads(l) for l in r.stderr.splitlines() if l.startswith("{")]
    timed = runs[warmup:]
    secs = sum(x["seconds"] for x in timed)
    samples = sum(x["samples"] for x in timed)
    # CPUMulticoreTracer runs min(hardware_concurrency()-1, maxThreads) tracer
    # threads; the last core spins its progress bar (cpuMulticore.cu:19-21,76-114).
    used = max(1, min(threads, (os.cpu_count() or 1) - 1))
    return samples / secs / 1e6, secs / max(len(timed), 1), used, samples // max(len(timed), 1)


def reference_window(desc, spp, max_bounce, win=None):
    """The reference's CPUMulticoreTracer::execute on all host threads over the
    pixel window win = (x0, y0, x1, y1) of desc's image (the whole image when
    None), through the profiler area the harness implements
    (cpuMulticore.cu:17).  Scene load and BVH build are not timed.  Returns
    (samples, seconds, threads used)."""
    import oracle
    from cuda_raytracer_b200 import scenes
    threads = os.cpu_count() or 1
    area = [str(v) for v in win] if win else []
    with tempfile.TemporaryDirectory() as tmp:
        path = scenes.write_scene(desc, tmp)
        r = subprocess.run([oracle.REF_BIN, "bench", os.path.basename(path), str(desc.width), str(desc.height),
                            str(spp), str(threads), str(max_bounce), "1", *area],
                           cwd=tmp, capture_output=True, text=True, timeout=1800, check=True)
    run_ = [json.loads(l) for l in r.stderr.splitlines() if l.startswith("{")][-1]
    # CPUMulticoreTracer runs min(hardware_concurrency()-1, maxThreads) tracer threads
    return run_["samples"], run_["seconds"], max(1, min(threads, threads - 1))


def layout_comparison(scene, desc, scene_json, n=4096, seed=5):
    """Bytes per closest-hit query in this build's layout and in the
    reference's, on the same rays: n camera rays at random pixels and, from
    each camera ray's hit, one cosine-distributed secondary ray.  Both use
    bytes = nodes x S_node + primitives x S_prim + 32 (ray in) + 16 (hit out):
    here wide nodes of 80 bytes and 48-byte primitive records (cr_trace_work);
    the reference's own walk (oracle/_ref/cr_ref work: Mesh::intersect's
    depth-first walk of each mesh's binary BVH, mesh.cu:200-267) reads 36-byte
    node records and 36-byte faces, and tests every sphere (16 bytes)."""
    import numpy as np
    import oracle
    from cuda_raytracer_b200 import scenes
    rng = np.random.default_rng(seed)
    px = np.stack([rng.integers(0, desc.width, n), rng.integers(0, desc.height, n)], 1)
    o, d = scenes.pinhole_rays(desc.camera, desc.width, desc.height, desc.spp, px, rng.integers(0, desc.spp, n))
    cam = np.concatenate([o, d, np.zeros((n, 1), np.float32)], 1).astype(np.float32)
    h = scene.trace(cam)
    sec = []
    groups = desc.groups
    for i in np.nonzero(h["prim"] >= 0)[0]:
        p_ = o[i].astype(np.float64) + d[i].astype(np.float64) * float(h["t"][i])
        pr = int(h["prim"][i])
        if pr < len(groups):
            g = groups[pr]
            v0, v1, v2 = (g.v[g.f[int(h["tri"][i])][k]].astype(np.float64) for k in range(3))
            nrm = np.cross(v1 - v0, v2 - v0)
        else:
            nrm = p_ - np.asarray(desc.spheres[pr - len(groups)]["o"], np.float64)
        nrm /= np.linalg.norm(nrm)
        if np.dot(nrm, d[i]) > 0:
            nrm = -nrm
        # cosine-distributed direction about the normal
        u1, u2 = rng.random(), rng.random()
        r, phi = np.sqrt(u1), 2 * np.pi * u2
        t1 = np.cross(nrm, [1.0, 0, 0] if abs(nrm[0]) < 0.9 else [0, 1.0, 0])
        t1 /= np.linalg.norm(t1)
        t2 = np.cross(nrm, t1)
        w = r * np.cos(phi) * t1 + r * np.sin(phi) * t2 + np.sqrt(max(0.0, 1 - u1)) * nrm
        sec.append(np.concatenate([p_ + nrm * 1e-3, w, [0.0]]))
    rays = np.concatenate([cam, np.asarray(sec, np.float32).reshape(-1, 7)]).astype(np.float32)
    nodes, prims = scene.trace_work(rays)
    with tempfile.TemporaryDirectory() as tmp:
        rp = os.path.join(tmp, "rays.f32")
        rays.tofile(rp)
        r = subprocess.run([oracle.REF_BIN, "work", os.path.basename(scene_json), rp], cwd=os.path.dirname(scene_json),
                           capture_output=True, text=True, timeout=1800, check=True)
    ref = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    m = len(rays)
    ours = (nodes * NODE_BYTES + prims * TRI_BYTES) / m + RAY_BYTES
    theirs = (ref["nodes"] * 36 + ref["faces"] * 36 + ref["spheres"] * 16) / m + RAY_BYTES
    return {"sample": f"{n} camera rays at random pixels and {m - n} cosine secondary rays from their hits",
            "ours": {"nodes_per_ray": round(nodes / m, 3), "prims_per_ray": round(prims / m, 3),
                     "bytes_per_ray": round(ours, 1), "layout": "80-byte wide nodes, 48-byte primitives"},
            "reference": {"node_records_per_ray": round(ref["nodes"] / m, 2), "faces_per_ray": round(ref["faces"] / m, 2),
                          "sphere_tests_per_ray": round(ref["spheres"] / m, 2), "bytes_per_ray": round(theirs, 1),
                          "layout": "36-byte binary nodes, 36-byte faces (its own BVH walk, counted by oracle/_ref/cr_ref work)"},
            "ratio": round(theirs / ours, 2)}


def reference_config0(repeats=3):
    """The reference's CPUMulticoreTracer::execute on the whole small box scene
    (256x256 at 64 spp, depth 8, 20 triangles + 2 spheres): the one
    configuration it renders in full within seconds, so that both arms time
    the identical workload.  Returns the line's config0 section."""
    from cuda_raytracer_b200 import scenes
    with tempfile.TemporaryDirectory() as tmp:
        d = scenes.config0()
        path = scenes.write_scene(d, tmp)
        rate, sec, cores, samples = reference_rate(path, repeats - 1, 1, d.spp, width=d.width, height=d.height)
    return {"workload": C0_WORKLOAD, "msamples_per_s": round(rate, 4), "ms_per_render": round(sec * 1e3, 2),
            "samples_per_render": samples, "cores": cores, "renders_timed": repeats - 1,
            "kind": "reference", "same_config": True}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/cr_ref was not built (make -C oracle ref)"}))
        return
    load_pkg()
    c0 = reference_config0()
    with tempfile.TemporaryDirectory() as tmp:
        _, path = make_workload(tmp)
        rate, sec, cores, samples = reference_rate(path, args.steps, args.warmup, args.ref_spp)
    sample = f"{WIDTH}x{HEIGHT} at {args.ref_spp} spp per step ({samples} paths), same scene and depth"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(rate, 4), "unit": "Msamples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": {"workload": "config1: 1024x768x256spp, 1.31M-tri displaced icosphere in the box, depth 8",
                   "sample_per_step": sample},
        "cpu_baseline": {"value": round(rate, 4), "unit": "Msamples/s", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(rate, 4), "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "config0": c0,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------- our arm
def guided_vs_plain(cr, dev, tmax_s, ref_spp, target=1e-3, l2_gbs=None, with_reference=False):
    """Time to relMSE <= target, plain MIS vs learned guiding, on the
    occluded-light scene (1024x1024, ~492k triangles, max depth 8).

    relMSE = mean over pixels and channels of ((I - R)^2 - Var[R]) / (R^2 + 1e-2),
    R a plain MIS render of ref_spp samples per pixel (Var[R] its per-pixel
    variance of the mean, removed so that the figure estimates the error
    against the converged image).  Each run renders 4 spp per call into one
    film; its clock is the device time of all its calls (CUDA events).  A run
    stops at the target or after tmax_s.

    Two plain runs: with the reference's Russian roulette (after bounce 3,
    the library's default for plain renders) and without roulette; the
    speed-up is taken against the faster of the two.  The guided run uses the
    library's defaults for guided renders (no roulette, every vertex but the
    last guided, 600 training steps front-loaded at 64 per wave); its guide
    first trains to its budget on 2-spp scratch passes (cr_guide_train,
    clocked), so that the measured film holds only samples of the trained
    guide."""
    import torch
    from cuda_raytracer_b200 import scenes
    res = 1024
    d = scenes.config3(width=res, height=res)
    sc = cr.Scene.from_desc(d)
    n = res * res
    stream = torch.cuda.current_stream(dev).cuda_stream

    def film():
        return (torch.zeros(n * 3, dtype=torch.float64, device=dev), torch.zeros(n * 3, dtype=torch.float64, device=dev),
                torch.zeros(n, dtype=torch.int32, device=dev))

    def render(f, spp, seed, guiding, rr_start=0):
        desc = cr.render_desc(res, res, spp, max_bounce=MAX_BOUNCE, estimator=cr.MIS, seed=seed, guiding=guiding,
                              rr_start=rr_start)
        sc.render_device(desc, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), stream=stream, stats=False)

    R = film()
    for i in range(ref_spp // 64):
        render(R, 64, 1_000_000 + i, False)
    torch.cuda.synchronize(dev)
    cnt = R[2].double().repeat_interleave(3)
    Rm = R[0] / cnt
    Rvar = (R[1] / cnt - Rm * Rm).clamp_min(0) / cnt
    den = Rm * Rm + 1e-2
    del R

    def timed(f, seed, guiding, rr_start):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        render(f, 4, seed, guiding, rr_start)
        e1.record()
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1)

    def run(guiding, rr_start=0):
        ms, k, train_ms = 0.0, 0, 0.0
        if guiding:
            # cr_guide_train: passes of 1024 x 1024 x 2 paths, the 64 x 32,768
            # paths a wave records, so every path rendered for training is used
            g = cr.Guide(sc).reset(seed=7)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            k = g.train(cr.render_desc(res, res, 1, max_bounce=MAX_BOUNCE, estimator=cr.MIS, seed=500_000,
                                       guiding=True, rr_start=rr_start), stream=stream)
            e1.record()
            torch.cuda.synchronize(dev)
            ms = train_ms = e0.elapsed_time(e1)
        F = film()
        spp, hit, err = 0, None, None
        while ms < tmax_s * 1e3:
            ms += timed(F, 1 + k, guiding, rr_start)
            spp += 4
            k += 1
            c2 = F[2].double().repeat_interleave(3)
            err = (((F[0] / c2 - Rm) ** 2 - Rvar) / den).mean().item()
            if err <= target:
                hit = ms / 1e3
                break
        return {"time_to_target_s": None if hit is None else round(hit, 3), "spp": spp,
                "training_s": round(train_ms / 1e3, 3), "relmse_at_stop": float(f"{err:.4e}"),
                "device_s": round(ms / 1e3, 3), "msamples_per_s": round(n * spp / ((ms - train_ms) / 1e3) / 1e6, 2)}

    plain = run(False)
    plain_no_rr = run(False, rr_start=MAX_BOUNCE + 1)
    guided = run(True)
    g = cr.Guide(sc)
    # the guide's inference kernel (k_guide_infer) on the trained guide: one
    # 4-spp guided render with stage timing gives its launches, rows and time
    F = film()
    st = sc.render_device(cr.render_desc(res, res, 4, max_bounce=MAX_BOUNCE, estimator=cr.MIS, seed=777_777,
                                         guiding=True), F[0].data_ptr(), F[1].data_ptr(), F[2].data_ptr(),
                          stream=stream)
    torch.cuda.synchronize(dev)
    del F
    launches = max(st.guide_launches, 1)
    infer_ms = max(st.ms_guide - st.ms_guide_train, 1e-6) / launches
    rows = st.guide_rows / launches
    tflops = rows * GUIDE_FLOPS_PER_ROW / (infer_ms / 1e3) / 1e12
    sector_gbs = rows * GUIDE_GATHERS_PER_ROW * 32 / (infer_ms / 1e3) / 1e9
    bf16, bf16_kind = measured_bf16()
    gtraffic = profiled_traffic("k_guide_infer_traffic.json")
    roofline = None if st.guide_launches == 0 else {
                "kernel": "k_guide_infer", "bound": "l2 (hash-grid gathers)", "launches": st.guide_launches,
                "rows_per_launch": round(rows), "launch_ms": round(infer_ms, 4),
                "traffic": round(gtraffic["dram_bytes_per_row"] * rows) if gtraffic else None,
                "traffic_note": ("ncu DRAM bytes per row over the 7 inference launches of one captured 4-spp guided "
                                 "render of this scene (profiles/k_guide_infer_traffic.json), scaled to this run's "
                                 "rows per launch") if gtraffic else None,
                "ms_per_4spp_render": round(st.ms_total, 2), "ms_guide_per_4spp_render": round(st.ms_guide, 2),
                "tensor": {"achieved": round(tflops, 2), "peak": bf16, "unit": "TFLOP/s", "frac": round(tflops / bf16, 4),
                           "peak_source": bf16_kind,
                           "flops_per_unit": f"{GUIDE_FLOPS_PER_ROW} per row (5 BF16 layers of 64 x 64)"},
                "l2": {"achieved": round(sector_gbs, 1), "peak": round(l2_gbs, 1) if l2_gbs else None, "unit": "GB/s",
                       "frac": round(sector_gbs / l2_gbs, 4) if l2_gbs else None,
                       "peak_source": "measured in this run (cr_measure_peaks: 32 MB L2-resident reads)",
                       "bytes_per_unit": f"{GUIDE_GATHERS_PER_ROW} random 8-byte hash-grid gathers per row (FP16 "
                                         "feature pairs of 12 levels x 4 cell edges), counted as the 32-byte "
                                         "sectors they touch"}}
    best = [x["time_to_target_s"] for x in (plain, plain_no_rr) if x["time_to_target_s"]]
    out = {"workload": "config3: occluded light (wall with a 0.4x0.4 aperture), 1024x1024, "
                       f"{sc.info()['triangles']} triangles, max depth 8, MIS estimator",
           "metric": f"device seconds to relMSE <= {target:g} against a {ref_spp}-spp plain reference",
           "reference_spp": ref_spp, "max_seconds": tmax_s, "plain": plain, "plain_no_roulette": plain_no_rr,
           "guided": guided,
           "guide": {"steps": g.info()["step"], **{k: v for k, v in g.configure().items()}, "roulette": "none"},
           "speedup": (round(min(best) / guided["time_to_target_s"], 3)
                       if best and guided["time_to_target_s"] else None),
           "speedup_vs_plain_reference_roulette": (round(plain["time_to_target_s"] / guided["time_to_target_s"], 3)
                                                   if plain["time_to_target_s"] and guided["time_to_target_s"] else None),
           "roofline": roofline}
    if with_reference:
        import oracle
        if oracle.ref_available():
            samples, secs, cores = reference_window(d, 1, MAX_BOUNCE)
            out["cpu_baseline"] = {"value": round(samples / secs / 1e6, 4), "unit": "Msamples/s", "cores": cores,
                                   "kind": "reference",
                                   "sample": f"the whole {res}x{res} image at 1 spp with the reference's own "
                                             "estimator (it has no MIS or guiding), same scene and depth; scene "
                                             "load and BVH build excluded"}
    sc.close()
    return out


def config0_section(cr, dev, steps, warmup, l2_gbs, with_reference):
    """The small box scene at its full configuration (256x256, 64 spp, depth 8,
    reference estimator), the workload both arms run identically.  Device
    throughput over `steps` renders (CUDA events, L2 flushed between renders),
    end to end through the public API from host arrays (scene upload, GPU BVH
    build, render, film to host), the closest-hit kernel's bandwidth against
    the in-run L2 read peak (the whole scene, 6 KB of nodes and triangles,
    lives in L2), and the reference CPU tracer on the same full render."""
    import numpy as np
    import torch
    from cuda_raytracer_b200 import scenes
    d = scenes.config0()
    W, H, spp = d.width, d.height, d.spp
    sc = cr.Scene.from_desc(d)
    n = W * H
    f = [torch.zeros(n * 3, dtype=torch.float64, device=dev), torch.zeros(n * 3, dtype=torch.float64, device=dev),
         torch.zeros(n, dtype=torch.int32, device=dev)]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    tune = sc.autotune(cr.render_desc(W, H, spp, max_bounce=MAX_BOUNCE, estimator=cr.KOISHI, seed=99),
                       stream=stream.cuda_stream).as_dict()

    def render(seed, stats=True, count=False):
        rd = cr.render_desc(W, H, spp, max_bounce=MAX_BOUNCE, estimator=cr.KOISHI, seed=seed, count_work=count)
        return sc.render_device(rd, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), stream=stream.cuda_stream,
                                stats=stats)

    for w in range(warmup):
        render(300 + w)
    cst = render(4242, count=True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    tot = {"extend": 0.0, "ext_launches": 0, "launches": 0, "samples": 0}
    torch.cuda.synchronize(dev)
    for k in range(steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        st = render(500 + k)
        ev[k][1].record(stream)
        tot["extend"] += st.ms_extend
        tot["ext_launches"] += st.extend_launches
        tot["launches"] += st.launches
        tot["samples"] += st.samples
    torch.cuda.synchronize(dev)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    ext_bytes = (cst.nodes * NODE_BYTES + cst.tris * TRI_BYTES + cst.rays_extend * RAY_BYTES) / max(cst.extend_launches, 1)
    ext_ms = tot["extend"] / max(tot["ext_launches"], 1)
    achieved = ext_bytes / (ext_ms / 1e3) / 1e9
    times = []
    for k in range(3):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        s2 = cr.Scene.from_desc(d)
        film, _ = s2.render(W, H, spp, max_bounce=MAX_BOUNCE, estimator=cr.KOISHI, seed=77 + k,
                            **{k2: tune[k2] for k2 in ("wave_paths", "refill_min", "traverse_blocks_per_sm", "shade_threads", "bin_rays", "shadow_vote", "shadow_refill_min")})
        s2.close()
        times.append(time.perf_counter() - t0)
        assert np.isfinite(film).all()
    e2e_ms = statistics.mean(times[1:]) * 1e3
    out = {"workload": C0_WORKLOAD, "msamples_per_s": round(tot["samples"] / ms / 1e3, 3),
           "ms_per_render": round(ms / steps, 3), "renders_timed": steps, "launches_per_render": tot["launches"] // steps,
           "e2e": {"msamples_per_s": round(n * spp / e2e_ms / 1e3, 3), "ms_per_render": round(e2e_ms, 2),
                   "h2d_bytes": int(sum(g.v.nbytes + g.n.nbytes + g.f.nbytes for g in d.groups)),
                   "d2h_bytes": n * 3 * 8, "includes": "scene upload, GPU BVH build, render, film copy to host"},
           "roofline": {"bound": "l2", "kernel": "k_extend", "achieved": round(achieved, 1), "peak": round(l2_gbs, 1),
                        "unit": "GB/s", "frac": round(achieved / l2_gbs, 4),
                        "peak_source": "measured in this run (cr_measure_peaks: 32 MB L2-resident reads)",
                        "algorithmic_bytes_per_launch": round(ext_bytes), "launch_ms": round(ext_ms, 4),
                        "nodes_per_ray": round(cst.nodes / max(cst.rays_extend, 1), 3),
                        "tris_per_ray": round(cst.tris / max(cst.rays_extend, 1), 3)},
           "autotuned": tune}
    if with_reference:
        import oracle
        if oracle.ref_available():
            ref = reference_config0()
            out["cpu_baseline"] = {"value": ref["msamples_per_s"], "unit": "Msamples/s", "cores": ref["cores"],
                                   "kind": "reference", "sample": "the whole configuration (256x256 at 64 spp), "
                                                                  f"{ref['renders_timed']} timed renders"}
            out["same_config"] = True
            out["speedup_vs_reference"] = round(out["msamples_per_s"] / ref["msamples_per_s"], 1)
            out["e2e_speedup_vs_reference"] = round(out["e2e"]["msamples_per_s"] / ref["msamples_per_s"], 1)
    sc.close()
    del flush
    return out


def batched_workload(cr, dev, n_scenes, seed=2, l2_gbs=None, with_reference=False):
    """The batched workload: n_scenes seeded scenes (triangle counts
    log-uniform in [1e3, 2e6], square images log-uniform 128..1024, spp from
    {16..256}, 1-4 lights) rendered as one batch replayed from a CUDA graph,
    against one render call per scene with the same work.  Device time (CUDA
    events) of one replay, after an autotune and a warm-up replay."""
    import torch
    from cuda_raytracer_b200 import scenes
    t0 = time.perf_counter()
    descs = [scenes.config2(i, seed) for i in range(n_scenes)]
    scs = [cr.Scene.from_desc(d) for d in descs]
    t_build = time.perf_counter() - t0
    films = []
    for d in descs:
        n = d.width * d.height
        films.append((torch.zeros(n * 3, dtype=torch.float64, device=dev), torch.zeros(n * 3, dtype=torch.float64, device=dev),
                      torch.zeros(n, dtype=torch.int32, device=dev)))
    jobs = [(sc, d.width, d.height, d.spp, 1 + i, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr())
            for i, (sc, d, f) in enumerate(zip(scs, descs, films))]
    total = sum(d.width * d.height * d.spp for d in descs)
    b = cr.Batch(jobs, max_bounce=MAX_BOUNCE, estimator=cr.KOISHI)
    tune = b.autotune().as_dict()
    b.render(0, stats=True)  # capture + warm-up
    st = b.render(1, stats=True)
    stream = torch.cuda.current_stream(dev).cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for (sc, w, h, spp, sd, *_), f in zip(jobs, films):
        dd = cr.render_desc(w, h, spp, max_bounce=MAX_BOUNCE, estimator=cr.KOISHI, seed=sd + 2)
        sc.render_device(dd, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), stream=stream, stats=False)
    e1.record()
    torch.cuda.synchronize(dev)
    ms_single = e0.elapsed_time(e1)
    # closest-hit roofline over the batch's scenes: per scene, a timed pass and
    # a counting pass over the same rays (spp / 16, same seed); the graph's
    # replay carries no per-kernel timing, and its traversal is the same
    # kernel over queues that mix the scenes' rays
    ext_ms, ext_bytes, ext_launches = 0.0, 0.0, 0
    for (sc, w, h, spp, sd, *_), f in zip(jobs, films):
        kw = dict(max_bounce=MAX_BOUNCE, estimator=cr.KOISHI, seed=sd + 3)
        sp = max(1, spp // 16)
        st_t = sc.render_device(cr.render_desc(w, h, sp, **kw), f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(),
                                stream=stream)
        st_c = sc.render_device(cr.render_desc(w, h, sp, count_work=True, **kw), f[0].data_ptr(), f[1].data_ptr(),
                                f[2].data_ptr(), stream=stream)
        ext_ms += st_t.ms_extend
        ext_launches += st_t.extend_launches
        ext_bytes += st_c.nodes * NODE_BYTES + st_c.tris * TRI_BYTES + st_c.rays_extend * RAY_BYTES
    achieved = ext_bytes / (ext_ms / 1e3) / 1e9
    hbm, hbm_kind = measured_peaks()
    roofline = {"bound": "l2", "kernel": "k_extend (per-scene passes over the batch's scenes at spp / 16)",
                "achieved": round(achieved, 1), "peak": round(l2_gbs, 1) if l2_gbs else None, "unit": "GB/s",
                "frac": round(achieved / l2_gbs, 4) if l2_gbs else None,
                "peak_source": "measured in this run (cr_measure_peaks: 32 MB L2-resident reads)",
                "hbm": {"peak": hbm, "frac": round(achieved / hbm, 4), "peak_source": hbm_kind},
                "launches": ext_launches, "launch_ms": round(ext_ms / max(ext_launches, 1), 4),
                "algorithmic_bytes": round(ext_bytes)}
    out = {"workload": f"config2: {n_scenes} scenes, {sum(d.n_triangles for d in descs)} triangles, "
                       f"{total} samples per replay, depth 8, reference estimator",
           "msamples_per_s": round(total / st.ms_total / 1e3, 2), "ms_per_replay": round(st.ms_total, 2),
           "per_scene_calls_msamples_per_s": round(total / ms_single / 1e3, 2),
           "speedup_vs_per_scene_calls": round(ms_single / st.ms_total, 3),
           "graph_nodes": st.graph_nodes, "kernel_launches_per_replay": st.launches, "waves": st.waves,
           "autotuned": tune,
           "scene_build_s": round(t_build, 1),
           "roofline": roofline}
    b.close()
    if with_reference:
        import oracle
        if oracle.ref_available():
            # every 8th scene, its central 32 x 32 window at the scene's own spp
            samples, secs, cores, t1 = 0, 0.0, 1, time.perf_counter()
            picked = list(range(0, n_scenes, 8))
            for i in picked:
                d = descs[i]
                x0, y0 = d.width // 2 - 16, d.height // 2 - 16
                n_, s_, cores = reference_window(d, d.spp, MAX_BOUNCE, (x0, y0, x0 + 32, y0 + 32))
                samples, secs = samples + n_, secs + s_
            out["cpu_baseline"] = {"value": round(samples / secs / 1e6, 4), "unit": "Msamples/s", "cores": cores,
                                   "kind": "reference",
                                   "sample": f"scenes {picked} of the batch, each its central 32x32 window at its "
                                             f"own spp through the reference's profiler area ({samples} paths, "
                                             f"{secs:.1f} s of rendering; scene load and BVH build excluded, "
                                             f"{time.perf_counter() - t1:.0f} s wall in all)"}
    return out


def window_time_to_target(cr, scene, W, H, win, max_bounce, ref_spp, tmax_s, dev, step_spp=16, target=1e-3):
    """Plain vs guided MIS time to relMSE <= target on the pixel window `win`
    (x0, y0, x1, y1) of a W x H frame: the reference is a plain MIS render of
    the window at ref_spp; each run renders step_spp per call into one film,
    clocked by CUDA events, until the target or tmax_s (relMSE as in
    guided_vs_plain, the reference's own variance removed).  The guided run
    first trains its guide to the budget on scratch passes of the window
    (cr_guide_train, clocked)."""
    import torch
    x0, y0, x1, y1 = win
    n = (x1 - x0) * (y1 - y0)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def film():
        return (torch.zeros(n * 3, dtype=torch.float64, device=dev), torch.zeros(n * 3, dtype=torch.float64, device=dev),
                torch.zeros(n, dtype=torch.int32, device=dev))

    def render(f, spp, seed, guiding):
        d = cr.render_desc(W, H, spp, max_bounce=max_bounce, estimator=cr.MIS, seed=seed, guiding=guiding, window=win)
        scene.render_device(d, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), stream=stream, stats=False)

    R = film()
    for i in range(ref_spp // 64):
        render(R, 64, 2_000_000 + i, False)
    torch.cuda.synchronize(dev)
    cnt = R[2].double().repeat_interleave(3)
    Rm = R[0] / cnt
    Rvar = (R[1] / cnt - Rm * Rm).clamp_min(0) / cnt
    den = Rm * Rm + 1e-2
    del R

    def run(guiding):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms, spp, k, hit, err, train_ms = 0.0, 0, 0, None, None, 0.0
        if guiding:  # train the guide to its budget on scratch passes of the window first (clocked)
            g = cr.Guide(scene).reset(seed=7)
            e0.record()
            k = g.train(cr.render_desc(W, H, 1, max_bounce=max_bounce, estimator=cr.MIS, seed=500_000, guiding=True,
                                       window=win), stream=stream)
            e1.record()
            torch.cuda.synchronize(dev)
            ms = train_ms = e0.elapsed_time(e1)
        F = film()
        while ms < tmax_s * 1e3:
            e0.record()
            render(F, step_spp, 1 + k, guiding)
            e1.record()
            torch.cuda.synchronize(dev)
            ms += e0.elapsed_time(e1)
            spp += step_spp
            k += 1
            c2 = F[2].double().repeat_interleave(3)
            err = (((F[0] / c2 - Rm) ** 2 - Rvar) / den).mean().item()
            if err <= target:
                hit = ms / 1e3
                break
        return {"time_to_target_s": None if hit is None else round(hit, 3), "spp": spp,
                "training_s": round(train_ms / 1e3, 3), "relmse_at_stop": float(f"{err:.4e}"),
                "device_s": round(ms / 1e3, 3), "msamples_per_s": round(n * spp / ((ms - train_ms) / 1e3) / 1e6, 2)}

    plain = run(False)
    guided = run(True)
    return {"window": list(win), "reference_spp": ref_spp, "max_seconds": tmax_s, "target": target,
            "roulette": {"plain": "after bounce 3", "guided": "none"}, "plain": plain, "guided": guided,
            "speedup": (round(plain["time_to_target_s"] / guided["time_to_target_s"], 3)
                        if plain["time_to_target_s"] and guided["time_to_target_s"] else None)}


C4_WINDOW = (1760, 990, 2080, 1170)  # the central 320x180 pixels of the 3840x2160 frame


def config4_section(cr, dev, steps, warmup, with_reference, ttt_seconds=40.0):
    """The large combined run: 21M triangles (16 instances of 4 displaced
    1.31M-triangle meshes under random rigid transforms, flattened into one
    BVH), 6 lights, 3840x2160, depth 12, MIS.  A step is 16 spp of the full
    image (1024 spp would take a minute per step).  Plain and guided
    Msamples/s (CUDA events, L2 flushed between steps), the closest-hit
    roofline against HBM (the 1.3 GB BVH and triangles exceed L2), time to
    relMSE 1e-3 on the central 320x180 window (a converged reference of the
    whole 4K frame would take hours), and the reference's CPU tracer on that
    window through its profiler area."""
    import torch
    from cuda_raytracer_b200 import scenes
    W4, H4, SPP4, MB4 = 3840, 2160, 16, 11
    t0 = time.perf_counter()
    desc = scenes.config4()
    scene = cr.Scene.from_desc(desc)
    build_s = time.perf_counter() - t0
    info = scene.info()
    npx = W4 * H4
    s = torch.zeros(npx * 3, dtype=torch.float64, device=dev)
    q = torch.zeros(npx * 3, dtype=torch.float64, device=dev)
    c = torch.zeros(npx, dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    tune = scene.autotune(cr.render_desc(W4, H4, SPP4, max_bounce=MB4, estimator=cr.MIS, seed=99),
                          stream=stream.cuda_stream).as_dict()

    def run(guiding, label):
        for w in range(warmup):
            d = cr.render_desc(W4, H4, SPP4, max_bounce=MB4, estimator=cr.MIS, seed=500 + w, guiding=guiding)
            scene.render_device(d, s.data_ptr(), q.data_ptr(), c.data_ptr(), stream=stream.cuda_stream, stats=False)
        torch.cuda.synchronize(dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        tot = {"extend": 0.0, "launches": 0, "ext_launches": 0, "samples": 0, "guide": 0.0, "rays": 0}
        clocks = ClockSampler(dev.index or 0)
        clocks.start()
        for k in range(steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            d = cr.render_desc(W4, H4, SPP4, max_bounce=MB4, estimator=cr.MIS, seed=900 + k, guiding=guiding)
            st = scene.render_device(d, s.data_ptr(), q.data_ptr(), c.data_ptr(), stream=stream.cuda_stream)
            ev[k][1].record(stream)
            tot["extend"] += st.ms_extend
            tot["launches"] += st.launches
            tot["ext_launches"] += st.extend_launches
            tot["samples"] += st.samples
            tot["guide"] += st.ms_guide
            tot["rays"] += st.rays_extend + st.rays_shadow
        torch.cuda.synchronize(dev)
        clk = clocks.stop()
        ms = sum(a.elapsed_time(b) for a, b in ev)
        return {"label": label, "msamples_per_s": round(tot["samples"] / ms / 1e3, 3),
                "mrays_per_s": round(tot["rays"] / ms / 1e3, 2), "ms_per_step": round(ms / steps, 2),
                "ms_guide_per_step": round(tot["guide"] / steps, 2), "launches": tot["launches"],
                "extend_ms_per_launch": round(tot["extend"] / max(tot["ext_launches"], 1), 4), "clocks": clk}

    plain = run(False, "plain MIS")
    cr.Guide(scene).reset(seed=7)
    guided = run(True, "guided MIS (tensor-core guide, online training)")
    dcount = cr.render_desc(W4, H4, 4, max_bounce=MB4, estimator=cr.MIS, seed=4242, count_work=True)
    cst = scene.render_device(dcount, s.data_ptr(), q.data_ptr(), c.data_ptr(), stream=stream.cuda_stream)
    ext_bytes = cst.nodes * NODE_BYTES + cst.tris * TRI_BYTES + cst.rays_extend * RAY_BYTES
    # bytes of a launch at 16 spp: the counting pass ran 4 spp with the same wave size
    ext_launch_bytes = ext_bytes / max(cst.extend_launches, 1)
    achieved = ext_launch_bytes / (plain["extend_ms_per_launch"] / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic("k_extend_traffic_config4.json")
    del s, q, c, flush
    torch.cuda.empty_cache()
    ttt = window_time_to_target(cr, scene, W4, H4, C4_WINDOW, MB4, 32768, ttt_seconds, dev)
    out = {"workload": "config4: 16 instances of 4 displaced icospheres (level 8) under random rigid transforms in "
                       "one BVH, 6 lights, 3840x2160, depth 12, MIS estimator, 16 spp per step",
           "triangles": info["triangles"], "bvh_nodes": info["bvh_nodes"], "scene_build_s": round(build_s, 1),
           "autotuned": tune, "plain": plain, "guided": guided,
           "roofline": {"bound": "hbm", "kernel": "k_extend (plain MIS steps)", "achieved": round(achieved, 1),
                        "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                        "traffic": (round(traffic["dram_bytes_per_ray"] * cst.rays_extend / max(cst.extend_launches, 1))
                                    if traffic else None),
                        "traffic_note": ("ncu DRAM bytes per ray over the closest-hit launches of one captured 1-spp "
                                         "render (profiles/k_extend_traffic_config4.json), scaled to this run's rays "
                                         "per launch")
                                        if traffic else None,
                        "algorithmic_bytes_per_launch": round(ext_launch_bytes),
                        "nodes_per_ray": round(cst.nodes / max(cst.rays_extend, 1), 3),
                        "tris_per_ray": round(cst.tris / max(cst.rays_extend, 1), 3)},
           "time_to_relmse": ttt,
           "note": "time to relMSE 1e-3 measured on the central 320x180 window against a 32768-spp plain reference "
                   "of that window (a converged reference of the full 4K frame would take hours)"}
    if with_reference:
        import oracle
        if oracle.ref_available():
            with tempfile.TemporaryDirectory() as tmp:
                path = scenes.write_scene(desc, tmp)
                threads = os.cpu_count() or 1
                x0, y0, x1, y1 = C4_WINDOW
                t1 = time.perf_counter()
                r = subprocess.run([oracle.REF_BIN, "bench", os.path.basename(path), str(W4), str(H4), "4",
                                    str(threads), str(MB4), "1", str(x0), str(y0), str(x1), str(y1)],
                                   cwd=tmp, capture_output=True, text=True, timeout=1800, check=True)
                wall = time.perf_counter() - t1
            run_ = [json.loads(l) for l in r.stderr.splitlines() if l.startswith("{")][-1]
            out["cpu_baseline"] = {"value": round(run_["samples"] / run_["seconds"] / 1e6, 4), "unit": "Msamples/s",
                                   "cores": max(1, min(threads, threads - 1)), "kind": "reference",
                                   "sample": f"the central {x1 - x0}x{y1 - y0} window at 4 spp through the "
                                             "reference's profiler area (reference estimator, same scene and depth; "
                                             f"scene load and BVH build excluded, {wall:.0f} s wall in all)"}
    scene.close()
    return out


def run_config4(args):
    """--workload config4: the large combined run alone, as one JSON line with
    guided Msamples/s as its value."""
    import torch
    cr = load_pkg()
    dev = torch.device("cuda", 0)
    c4 = config4_section(cr, dev, args.steps, args.warmup, not args.no_cpu_baseline)
    g = c4["guided"]
    line = {
        "metric": "Msamples/s, guided MIS, 3840x2160 at 16 spp per step, 21M-triangle instanced scene, depth 12",
        "value": g["msamples_per_s"], "unit": "Msamples/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": g["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene, no dataset)",
        "config": {"workload": c4["workload"], "triangles": c4["triangles"], "bvh_nodes": c4["bvh_nodes"],
                   "l2": "flushed between timed steps (256 MB write)"},
        "roofline": c4["roofline"], "clocks": g["clocks"], "gpu_launches": g["launches"], "e2e": None,
        "cpu_baseline": c4.get("cpu_baseline"), "config4": c4,
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    cr = load_pkg()
    tmp = tempfile.mkdtemp()
    desc, path = make_workload(tmp)
    scene = cr.Scene.from_desc(desc)
    info = scene.info()
    spp = args.spp or SPP
    npx = WIDTH * HEIGHT
    s = torch.zeros(npx * 3, dtype=torch.float64, device=dev)
    q = torch.zeros(npx * 3, dtype=torch.float64, device=dev)
    c = torch.zeros(npx, dtype=torch.int32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    def step(seed, stats=True):
        d = cr.render_desc(WIDTH, HEIGHT, spp, max_bounce=MAX_BOUNCE, estimator=cr.KOISHI, seed=seed,
                           wave_paths=args.wave_paths)
        return scene.render_device(d, s.data_ptr(), q.data_ptr(), c.data_ptr(), stream=stream.cuda_stream,
                                   stats=stats)

    # launch configuration: autotuned on a sample band of the image (untimed)
    tuning = None
    if not args.no_autotune:
        td = cr.render_desc(WIDTH, HEIGHT, spp, max_bounce=MAX_BOUNCE, estimator=cr.KOISHI, seed=99)
        tuning = scene.autotune(td, stream=stream.cuda_stream).as_dict()
        torch.cuda.synchronize(dev)

    # warm-up
    for w in range(args.warmup):
        step(1000 + w)
    torch.cuda.synchronize(dev)

    # work counts for the roofline (untimed counting pass on one seed)
    dcount = cr.render_desc(WIDTH, HEIGHT, spp, max_bounce=MAX_BOUNCE, estimator=cr.KOISHI, seed=4242,
                            wave_paths=args.wave_paths, count_work=True)
    cst = scene.render_device(dcount, s.data_ptr(), q.data_ptr(), c.data_ptr(), stream=stream.cuda_stream)

    # timed region
    clocks = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    totals = {"extend": 0.0, "shadow": 0.0, "shade": 0.0, "other": 0.0, "launches": 0, "ext_launches": 0,
              "shadow_launches": 0,
              "rays_extend": 0, "rays_shadow": 0, "samples": 0}
    for k in range(args.steps):
        flush.fill_(float(k))  # L2 flush between timed steps (outside the events)
        ev[k][0].record(stream)
        st = step(replica_seed(rank, k))
        ev[k][1].record(stream)
        totals["extend"] += st.ms_extend
        totals["shadow"] += st.ms_shadow
        totals["shade"] += st.ms_shade
        totals["other"] += st.ms_other
        totals["launches"] += st.launches
        totals["ext_launches"] += st.extend_launches
        totals["shadow_launches"] += st.shadow_launches
        totals["rays_extend"] += st.rays_extend
        totals["rays_shadow"] += st.rays_shadow
        totals["samples"] += st.samples
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    value, ms_max, samples_all = job_throughput(ms, totals["samples"], dev, world)

    # roofline of the closest-hit kernel
    ext_bytes = cst.nodes * NODE_BYTES + cst.tris * TRI_BYTES + cst.rays_extend * RAY_BYTES
    ext_launch_bytes = ext_bytes / max(cst.extend_launches, 1)
    ext_launch_ms = totals["extend"] / max(totals["ext_launches"], 1)
    achieved = ext_launch_bytes / (ext_launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic()
    # L2-resident read bandwidth and FP32 FMA rate of this GPU, measured now:
    # the working set of this workload's traversal fits in L2
    l2_gbs, fp32_tflops = cr.measure_peaks(stream.cuda_stream)
    # random 80-byte node and 48-byte triangle gathers from an L2-resident
    # array of this workload's size (node + triangle records, 73 MB): the
    # achievable L2 rate for the traversal's access pattern; the kernel reads
    # nodes and triangles in about a 6:4 byte ratio
    ws = min(int(info["bvh_nodes"] * NODE_BYTES + info["triangles"] * TRI_BYTES), 100 << 20)
    g80 = cr.measure_gather(80, ws, stream.cuda_stream)
    g48 = cr.measure_gather(48, ws, stream.cuda_stream)
    ext_flops = (cst.nodes * 96 + cst.tris * 40) / max(cst.extend_launches, 1)  # 8 slab tests x 12 + 40 per triangle
    # the gather peak for this kernel's mix of node and triangle bytes (harmonic)
    nb, tb = cst.nodes * NODE_BYTES, cst.tris * TRI_BYTES
    gather_peak = (nb + tb) / (nb / g80 + tb / g48) if nb + tb > 0 else g80
    # any-hit launches: nodes x 80 B + triangles x 48 B + rays x 48 B (ray in, contribution)
    sh_bytes = (cst.shadow_nodes * NODE_BYTES + cst.shadow_tris * TRI_BYTES + cst.rays_shadow * 48) / max(cst.shadow_launches, 1)

    # end to end through the public API from host arrays
    e2e = None
    if rank == 0 and args.e2e_steps > 0:
        import numpy as np
        h2d = sum(g.v.nbytes + g.n.nbytes + g.f.nbytes for g in desc.groups)
        d2h = npx * 3 * 8 + npx * 4
        times = []
        # one untimed step first, as the device-timed steps have warm-up steps:
        # the first scene of a size maps the pool's memory for its wave state
        for k in range(-1, args.e2e_steps):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            sc2 = cr.Scene.from_desc(desc)
            tk = {k2: tuning[k2] for k2 in ("wave_paths", "refill_min", "traverse_blocks_per_sm", "shade_threads", "bin_rays", "shadow_vote", "shadow_refill_min")} if tuning else {}
            film, _ = sc2.render(WIDTH, HEIGHT, spp, max_bounce=MAX_BOUNCE, estimator=cr.KOISHI, seed=77 + k, **tk)
            sc2.close()
            if k >= 0:
                times.append(time.perf_counter() - t0)
            assert np.isfinite(film).all()
        e2e = {"value": round(npx * spp / statistics.mean(times) / 1e6, 4), "unit": "Msamples/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": round(statistics.mean(times) * 1e3, 3),
               "includes": "scene upload, GPU BVH build, render, film copy to host",
               "warmup_steps": 1}

    cpu = None
    layout = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            rate, sec, cores, samples = reference_rate(path, 1, 0, args.ref_spp)
            cpu = {"value": round(rate, 4), "unit": "Msamples/s", "cores": cores, "kind": "reference",
                   "sample": f"{WIDTH}x{HEIGHT} at {args.ref_spp} spp ({samples} paths) of the same scene, "
                             f"{sec:.1f} s of CPU time"}
            try:
                layout = layout_comparison(scene, desc, path)
            except (subprocess.SubprocessError, OSError, ValueError) as e:  # a checker failure must not stop the bench
                layout = {"unavailable": f"{type(e).__name__}: {e}"[:200]}
        else:
            cpu = {"value": None, "unit": "Msamples/s", "cores": 0, "kind": "reference",
                   "sample": "oracle/_ref/cr_ref not built"}

    c0 = None
    if rank == 0 and world == 1 and not args.no_config0:
        c0 = config0_section(cr, dev, 20, 3, l2_gbs, not args.no_cpu_baseline)

    guiding = None
    if rank == 0 and world == 1 and args.guide_seconds > 0:
        del s, q, c, flush
        torch.cuda.empty_cache()
        guiding = guided_vs_plain(cr, dev, args.guide_seconds, args.guide_ref_spp, l2_gbs=l2_gbs,
                                  with_reference=not args.no_cpu_baseline)
    batch = None
    if rank == 0 and world == 1 and args.batch_scenes > 0:
        batch = batched_workload(cr, dev, args.batch_scenes, l2_gbs=l2_gbs, with_reference=not args.no_cpu_baseline)
    c4 = None
    if rank == 0 and world == 1 and not args.no_config4:
        torch.cuda.empty_cache()
        c4 = config4_section(cr, dev, 2, 3, not args.no_cpu_baseline)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "Msamples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded procedural scene, no dataset)",
            "config": {"workload": "config1: 1024x768x256spp, 1.31M-tri displaced icosphere in the box, depth 8",
                       "triangles": info["triangles"], "bvh_nodes": info["bvh_nodes"], "spp": spp,
                       "estimator": "reference (koishi)", "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"replica-per-gpu x{world}", "autotuned": tuning},
            "mrays_per_s": round((totals["rays_extend"] + totals["rays_shadow"]) * world / (ms_max / 1e3) / 1e6, 2),
            "stage_ms_per_step": {k: round(totals[k] / args.steps, 3) for k in ("extend", "shadow", "shade", "other")},
            "roofline": {"bound": "hbm", "kernel": "k_extend", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                         "traffic": (round(traffic["dram_bytes_per_ray"] * cst.rays_extend / max(cst.extend_launches, 1))
                                     if traffic else None),
                         "traffic_note": ("ncu DRAM bytes per ray over the closest-hit launches of one captured 4-spp "
                                          "render (profiles/k_extend_traffic.json), scaled to this run's rays per "
                                          "launch") if traffic else None,
                         "algorithmic_bytes_per_launch": round(ext_launch_bytes),
                         "launch_ms": round(ext_launch_ms, 4),
                         "nodes_per_ray": round(cst.nodes / max(cst.rays_extend, 1), 3),
                         "tris_per_ray": round(cst.tris / max(cst.rays_extend, 1), 3),
                         "shadow": {"kernel": "k_shadow (any hit)",
                                    "rays_per_launch": round(cst.rays_shadow / max(cst.shadow_launches, 1)),
                                    "nodes_per_ray": round(cst.shadow_nodes / max(cst.rays_shadow, 1), 3),
                                    "tris_per_ray": round(cst.shadow_tris / max(cst.rays_shadow, 1), 3),
                                    "launch_ms": round(totals["shadow"] / max(totals["shadow_launches"], 1), 4),
                                    "achieved_gbs": round(sh_bytes / max(totals["shadow"] / max(totals["shadow_launches"], 1), 1e-9) / 1e6, 1)},
                         "l2": {"achieved": round(achieved, 1), "peak": round(l2_gbs, 1), "unit": "GB/s",
                                "frac": round(achieved / l2_gbs, 4),
                                "peak_source": "measured in this run (cr_measure_peaks: 32 MB L2-resident reads)"},
                         "l2_gather": {"achieved": round(achieved, 1), "peak": round(gather_peak, 1), "unit": "GB/s",
                                       "frac": round(achieved / gather_peak, 4),
                                       "peak_source": ("measured in this run (cr_measure_gather: random 80-byte "
                                                       f"node and 48-byte triangle records from an L2-resident "
                                                       f"{ws >> 20} MB array, {g80:.0f} and {g48:.0f} GB/s, "
                                                       "weighted by this kernel's node/triangle bytes)")},
                         "fp32": {"achieved": round(ext_flops / (ext_launch_ms / 1e3) / 1e12, 3),
                                  "peak": round(fp32_tflops, 2), "unit": "TFLOP/s",
                                  "frac": round(ext_flops / (ext_launch_ms / 1e3) / 1e12 / fp32_tflops, 4),
                                  "peak_source": "measured in this run (cr_measure_peaks: FMA chains)",
                                  "flops_per_unit": "96 per wide node (8 slab tests) + 40 per triangle test"},
                         "reference_layout": (layout if layout and "unavailable" in layout else
                                              dict(layout, gbs_at_this_ray_rate=round(
                             layout["reference"]["bytes_per_ray"] * cst.rays_extend / max(cst.extend_launches, 1)
                             / (ext_launch_ms / 1e3) / 1e9, 1)) if layout else None)},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk,
            "gpu_launches": totals["launches"],
            "config0": c0,
            "guiding": guiding,
            "batch": batch,
            "config4": c4,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def profile_case(name):
    """Small cases for the ncu captures summarised under profiles/ (a few GB on
    the device, seconds of GPU work).  Each render prints one JSON line with
    its stats, so that captured launches can be mapped to renders.

    guide_infer     the occluded-light scene at 1024x1024 with a fresh guide
                    (seed 7, the library's guiding defaults): five guided MIS
                    renders of 4 spp, one wave each.  The first wave trains
                    without sampling the guide; each later one runs
                    k_guide_infer on bounces 0-6.
    config4_extend  the large combined scene (21M triangles): one 1-spp MIS
                    render of the 3840x2160 image at max_bounce 11."""
    import torch
    cr = load_pkg()
    from cuda_raytracer_b200 import scenes
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    if name == "guide_infer":
        d = scenes.config3(width=1024, height=1024)
        renders = [cr.render_desc(1024, 1024, 4, max_bounce=MAX_BOUNCE, estimator=cr.MIS, seed=100 + k, guiding=True)
                   for k in range(5)]
    else:
        d = scenes.config4()
        renders = [cr.render_desc(3840, 2160, 1, max_bounce=11, estimator=cr.MIS, seed=4242)]
    sc = cr.Scene.from_desc(d)
    if name == "guide_infer":
        cr.Guide(sc).reset(seed=7)
    n = renders[0].width * renders[0].height
    f = [torch.zeros(n * 3, dtype=torch.float64, device=dev), torch.zeros(n * 3, dtype=torch.float64, device=dev),
         torch.zeros(n, dtype=torch.int32, device=dev)]
    for k, rd in enumerate(renders):
        st = sc.render_device(rd, f[0].data_ptr(), f[1].data_ptr(), f[2].data_ptr(), stream=stream)
        torch.cuda.synchronize(dev)
        print(json.dumps({"case": name, "render": k, "waves": st.waves, "extend_launches": st.extend_launches,
                          "rays_extend": st.rays_extend, "guide_launches": st.guide_launches,
                          "guide_rows": st.guide_rows, "ms_total": round(st.ms_total, 3),
                          "ms_guide": round(st.ms_guide, 3), "ms_guide_train": round(st.ms_guide_train, 3)}),
              flush=True)
    sc.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--spp", type=int, default=0, help="override spp per step (default: the workload's 256)")
    ap.add_argument("--wave-paths", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--ref-spp", type=int, default=4, help="spp of the reference's bounded CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-config0", action="store_true", help="skip the small box scene's section")
    ap.add_argument("--no-config4", action="store_true", help="skip the large combined run's section")
    ap.add_argument("--guide-seconds", type=float, default=25.0,
                    help="device-time cap of each guided/plain time-to-relMSE run (0: skip them)")
    ap.add_argument("--guide-ref-spp", type=int, default=4096)
    ap.add_argument("--batch-scenes", type=int, default=64, help="scenes of the batched workload (0: skip it)")
    ap.add_argument("--workload", choices=["config1", "config4"], default="config1",
                    help="config1: the headline 1024x768x256spp line; config4: the large combined run")
    ap.add_argument("--profile-case", choices=["guide_infer", "config4_extend"], default=None,
                    help="run one small case for an ncu capture (profiles/) and exit")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.profile_case:
        profile_case(args.profile_case)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "config4":
        run_config4(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
