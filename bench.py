"""NICP registration benchmark on B200 (one JSON line on stdout).

Workload (default): 640x480 frame-to-frame odometry over a seeded 200-frame
synthetic trajectory (fx = fy = 525, cx = 319.5, cy = 239.5; noise 0.0015 z^2,
2% dropped pixels).  One step = build all 200 clouds
(DepthImageConverterIntegralImage::compute) and align the 199 consecutive
pairs (AlignerProjective::align, reference defaults, 10 outer x 1 inner) in
one batched, graph-captured device loop.  Metric: 640x480 pairs/s.

  value        inputs already resident in HBM, CUDA events on the library stream
  e2e          through the public C ABI with pinned host frames: host->device
               copies of every frame and device->host of every pose inside the
               timed region
  plain_*      the one-pair-per-call path (nicp_cloud_from_depth_u16 +
               nicp_align per pair), for the batched/plain ratio
  roofline     the kernel with the largest share of device time, algorithmic
               bytes per launch / average launch time (CUDA events)
  cpu_baseline the reference algorithm restated in C++ (oracle REF32, all host
               threads) on a bounded sample of the same workload
  mixed_batch  512 independent pairs of mixed resolution, <= 20 x 2 iterations
               with early exit, batched vs the plain per-pair loop
  scene_fusion frames fused into one scene (Cloud::add + Merger::merge)
  nn_align     AlignerNN on 640x480 pairs (exact nearest-neighbour association)
  serving      the request loop (nicp_server_*) under open-loop Poisson load:
               64 camera streams, 30/60/10% 320x240/640x480/1280x720,
               p50/p99 latency and throughput per arrival rate

--impl reference runs only the CPU reference arm.  Multi-GPU (torchrun):
replicas only -- every rank runs the same workload on its own GPU; value is
the total over ranks divided by the slowest rank's time.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "640x480 NICP pairs/s (frame-to-frame, batched)"
HBM_FALLBACK = 6650.0


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def max_over_ranks_of(dist, x):
    """The slowest rank's time: every rank gets the maximum of x (gloo
    all-reduce over host tensors; `dist` is torch.distributed or None)."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, units_per_rank, steps, ms_max):
    """Whole-job throughput of `world` replicas: the units every rank
    processed, divided by the slowest rank's time."""
    return world * units_per_rank * steps / (ms_max / 1e3)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region.
    Started before the warm-up (so that nvidia-smi's own start-up is not
    inside the timed region); mark() brackets the timed region and stop()
    keeps the samples that arrived inside it (all of them if none did)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.reader = None
        self.window = [None, None]

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def mark(self, which):
        self.window[which] = time.monotonic()

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.reader.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = self.window
        lines = [ln for t, ln in self.lines if t0 is not None and t1 is not None and t0 <= t <= t1 + 0.25]
        if not lines:
            lines = [ln for _, ln in self.lines]
        for ln in lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ workload
def make_workload(seed, frames, cam_name="640x480", period=None):
    from nicp_b200 import synth
    imgs, poses, cam = synth.render_sequence(seed, cam_name, n_frames=frames, period=period)
    return np.stack(imgs), poses, cam


def gpu_objects(ctx, cam):
    from nicp_b200 import _lib as L
    from nicp_b200 import api
    proj = api.PinholePointProjector(ctx)
    proj.setCameraMatrix([[cam["fx"], 0, cam["cx"]], [0, cam["fy"], cam["cy"]], [0, 0, 1]])
    proj.setImageSize(cam["rows"], cam["cols"])
    conv = api.DepthImageConverterIntegralImage(proj, api.StatsCalculatorIntegralImage(),
                                                api.PointInformationMatrixCalculator(),
                                                api.NormalInformationMatrixCalculator())
    corr = api.CorrespondenceFinderProjective(ctx).params()
    lin = api.Linearizer(ctx).params()
    prm = L.AlignParams()
    ctx.lib.nicp_default_align_params(prm)
    prm.compute_statistics = 0  # the optional post-pass; not part of pairs/s
    return proj, conv, corr, lin, prm


def run_step(ctx, frames_ptrs, cam_c, prm_c, clouds, corr, lin, prm, on_device):
    from nicp_b200 import api
    n = len(clouds)
    api.build_batch(ctx, frames_ptrs, [cam_c] * n, prm_c, clouds, on_device=on_device)
    return api.align_batch(ctx, clouds[:-1], clouds[1:], [cam_c] * (n - 1), None, corr, lin, prm)


# Algorithmic bytes per unit (the per-stage figures of the scope table):
#   S1 unproject     2P + 4P + 12V          S2 moments   bands: 2P + 3 (10 s P / 16); sweep: 2P + 10 s P / 16 + 10 s P
#   S3 stats + Omega 10 s P + 6P + 28V      S4 z-buffer  16V (the point and its w, which carries the
#                    (+ 48V when the information matrices are written out:
#                    Stats kept or a general form; the headline leaves them
#                    implicit)
#                                                        "has a normal" bit of the key) + 8V atomics
#   S5 corr + lin    8P + 56 C: both index images, then per correspondence
#                    point xyz, normal xyz and curvature of both clouds; the
#                    information matrices are rebuilt from the current normal
#                    (structured Omega), not read (the general path adds 48 C)
#                    (s = 8 bytes per FP64 moment)
def build_bytes(P, V, s=8):
    """One frame build: S1 + band totals/carries + sweep + S3 (bytes)."""
    return (2 * P + 4 * P + 12 * V) + (2 * P + 3 * 10 * s * P / 16) + (2 * P + 10 * s * P / 16 + 10 * s * P) + \
        (10 * s * P + 6 * P + 28 * V)


def align_bytes(P, V, C, outer, inner):
    """One alignment: the current cloud's projection (points 16V, atomics 8V)
    and resolve (z-buffer read 8P, index write 4P, z-buffer reset 8P), then
    per outer iteration the reference projection (24V) and per inner iteration
    the fused pass: z-buffer read and reset (16P) + current index (4P) on the
    first, plus the reference index written (4P) when more follow; later
    inner iterations read both index images (8P); 56 bytes per accepted
    correspondence (points, normals, curvatures of both clouds)."""
    first = 20 * P + (4 * P if inner > 1 else 0) + 56 * C
    later = (inner - 1) * (8 * P + 56 * C)
    return 24 * V + 20 * P + outer * (24 * V + first + later)


def algorithmic_bytes(kernel, P, V, C, launches_per_step, pairs):
    s = 8
    if kernel == "unproject":
        return (2 * P + 4 * P + 12 * V) * pairs
    if kernel == "moments_bands":  # band totals (depth, totals write) + carries (read, write)
        return (2 * P + 3 * 10 * s * P / 16) * pairs
    if kernel == "moments_sweep":  # depth, carry rows, every integral value written once
        return (2 * P + 10 * s * P / 16 + 10 * s * P) * pairs
    if kernel == "stats_omega":
        return (10 * s * P + 6 * P + 28 * V) * pairs
    if kernel == "zbuffer":
        return (16 * V + 8 * V) * pairs
    if kernel == "corr_lin":
        return (20 * P + 56 * C) * pairs
    if kernel == "resolve":
        return (8 * P + 4 * P + 8 * P) * pairs
    return 0


def measured_traffic(kernel, units):
    """DRAM bytes of one launch of `kernel` processing `units` pairs or
    frames, from the committed ncu summary (None if it has no entry)."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_640x480_seq.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 3 and not line.startswith("#") and parts[0] == kernel:
                    return float(parts[2]) * units[parts[1]]
    except OSError:
        pass
    return None


def profile_step(ctx, run):
    """Per-kernel device time of one step (CUDA events on the library stream)."""
    from nicp_b200 import _lib as L
    ctx.set_profiling(True)
    ctx.synchronize()
    res = run()
    prof = {}
    for k in L.KERNELS:
        ms, n = ctx.read_profile(k)
        if n:
            prof[k] = (ms, n)
    ctx.set_profiling(False)
    return prof, res


def cpu_baseline(frames, cam, seconds=15.0, threads=None):
    """Oracle REF32 (the reference algorithm, float, reference order) on the
    host cores: build + align per frame pair until `seconds` elapse."""
    from oracle import oracle as O
    threads = threads or os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"])
    prm = O.align_params(threads=threads)
    t0 = time.perf_counter()
    prev, _ = O.build_cloud(O.REF32, frames[0], oc)
    pairs = 0
    k = 1
    while k < len(frames):
        cur, _ = O.build_cloud(O.REF32, frames[k], oc)
        O.align(O.REF32, prev, cur, oc, prm=prm)
        prev = cur
        pairs += 1
        k += 1
        if time.perf_counter() - t0 > seconds and pairs >= 2:
            break
    dt = time.perf_counter() - t0
    # the first frame's build is included in dt: amortised over the sample
    return pairs / dt, pairs, dt, threads


def pose_case(d1, d2, cam, T, outer=10, inner=1, eps=0.0, guess=None, truth=None):
    """One GPU pose to check: reference and current uint16 frames, camera
    dict, the GPU's pose, the loop controls, the initial guess and the truth."""
    return dict(d1=d1, d2=d2, cam=cam, T=np.asarray(T, float).reshape(4, 4), outer=outer, inner=inner, eps=eps,
                guess=None if guess is None else np.asarray(guess, float).reshape(4, 4), truth=truth)


def oracle_pose_check(cases, threads=None):
    """The checker: each case is run through the oracle's FP64 pipeline (the
    reference algorithm in double, from the same frames, the same guess and
    loop controls) and the GPU pose's distance to it is reported (radians,
    metres).  Where the truth is known, a case whose FP64 pose ends more than
    0.05 rad or 5 cm from it is an alignment the algorithm itself does not
    converge on; such cases are counted apart ("diverged") and kept out of
    the converged maxima.  A case outside 1e-5 rad / 0.05 mm is listed with
    how far the FP64 loop still moved in its last outer iteration (0 when it
    stopped on its own exit test) and how far the reference's own FP32
    pipeline (the REF32 oracle) ends from FP64 on it."""
    from oracle import oracle as O
    from nicp_b200 import synth
    threads = threads or os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    errs, diverged, outside = [], [], []
    for c in cases:
        cam = c["cam"]
        oc = O.camera(cam["rows"], cam["cols"], cam["fx"], cam["fy"], cam["cx"], cam["cy"],
                      max_distance=cam.get("max_distance", 6.0))
        a, _ = O.build_cloud(O.F64, c["d1"], oc)
        b, _ = O.build_cloud(O.F64, c["d2"], oc)
        prm = O.align_params(outer_iterations=c["outer"], inner_iterations=c["inner"], early_exit_eps=c["eps"])
        r = O.align(O.F64, a, b, oc, guess=c["guess"], prm=prm)
        e = synth.pose_error(c["T"], r["T"])
        if c["truth"] is not None:
            tr, tt = synth.pose_error(r["T"], c["truth"])
            if tr > 0.05 or tt > 0.05:
                diverged.append({"rad": float(e[0]), "m": float(e[1]), "f64_vs_truth_rad": float(tr)})
                continue
        errs.append(e)
        if e[0] > 1e-5 or e[1] > 5e-5:
            last = (0.0, 0.0)
            if r["outer_iterations_run"] >= c["outer"] and c["outer"] > 1:
                prm.outer_iterations = c["outer"] - 1
                last = synth.pose_error(r["T"], O.align(O.F64, a, b, oc, guess=c["guess"], prm=prm)["T"])
                prm.outer_iterations = c["outer"]
            a32, _ = O.build_cloud(O.REF32, c["d1"], oc)
            b32, _ = O.build_cloud(O.REF32, c["d2"], oc)
            q = synth.pose_error(O.align(O.REF32, a32, b32, oc, guess=c["guess"], prm=prm)["T"], r["T"])
            outside.append({"rad": float(e[0]), "m": float(e[1]), "f64_last_step_rad": float(last[0]),
                            "f64_last_step_m": float(last[1]), "ref32_vs_f64_rad": float(q[0]),
                            "ref32_vs_f64_m": float(q[1])})
    er = np.array([e[0] for e in errs]) if errs else np.zeros(1)
    et = np.array([e[1] for e in errs]) if errs else np.zeros(1)
    return {"pairs": len(errs), "rad_max": float(er.max()), "rad_p99": float(np.percentile(er, 99)),
            "rad_median": float(np.median(er)), "m_max": float(et.max()), "m_p99": float(np.percentile(et, 99)),
            "within_1e-5rad_0.05mm": int(np.sum((er <= 1e-5) & (et <= 5e-5))), "outside_1e-5rad_0.05mm": outside,
            "diverged": diverged}


def reference_arm(args, rank, world):
    if rank != 0:
        return 0
    # the first 40 frames of the same trajectory (same per-frame motion)
    frames, poses, cam = make_workload(args.seed, min(args.frames, 40), period=args.period or args.frames)
    for _ in range(max(0, args.warmup)):
        cpu_baseline(frames[:3], cam, seconds=0.0)
    vals, total_pairs, total_t = [], 0, 0.0
    per_step = min(args.cpu_seconds, 150.0 / max(1, args.steps))  # whole run stays within a few minutes
    for _ in range(args.steps):
        v, n, dt, threads = cpu_baseline(frames, cam, seconds=per_step)
        vals.append(v)
        total_pairs += n
        total_t += dt
    value = total_pairs / total_t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args),
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads, "kind": "port",
                             "sample": "%d frame pairs of the 640x480 sequence per step (build + align)" %
                                       (total_pairs // max(1, args.steps))},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ mixed batch leg
MIXED_CAMS = ("160x120", "320x240", "640x480")


def mixed_batch_leg(ctx, stream, device, seed, npairs=512, steps=3, warmup=3, plain_pairs=48):
    """512 independent frame pairs, each its own seeded scene, resolutions
    drawn uniformly from 160x120 / 320x240 / 640x480, the current frame
    offset by 0.5-5 deg and 1-8 cm.  One step builds the 1024 clouds and
    aligns the 512 pairs (up to 20 outer x 2 inner, a pair stops once its
    pose change falls below 1e-6) in one graph-captured device loop.  The
    plain leg runs the same pairs one call at a time (nicp_cloud_from_depth_u16
    twice + nicp_align), with the same iteration controls."""
    import ctypes as Cc
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from nicp_b200 import _lib as L
    from nicp_b200 import api, synth

    rng = np.random.default_rng(seed)
    names = [MIXED_CAMS[i] for i in rng.integers(0, 3, size=npairs)]
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        pairs = list(ex.map(lambda i: synth.render_pair(seed + 1000 + i, names[i], deg=0.5, deg_hi=5.0, meters=0.01,
                                                        m_hi=0.08), range(npairs)))
    # device-resident frames: one buffer, 256-byte aligned slots
    sizes = [2 * p[0].size for p in pairs for _ in range(2)]
    offs = np.concatenate([[0], np.cumsum([(s + 255) // 256 * 256 for s in sizes])])
    dev = torch.empty(int(offs[-1]), dtype=torch.uint8, device="cuda:%d" % device)
    host = torch.empty(int(offs[-1]), dtype=torch.uint8).pin_memory()
    hv = host.numpy()
    for k, (p, j) in enumerate((p, j) for p in pairs for j in range(2)):
        a = np.ascontiguousarray(p[j], np.uint16).view(np.uint8).ravel()
        hv[offs[k]:offs[k] + a.size] = a
    dev.copy_(host)
    cams = []
    for d1, d2, Tgt, cam in pairs:
        proj = api.PinholePointProjector(ctx)
        proj.setCameraMatrix([[cam["fx"], 0, cam["cx"]], [0, cam["fy"], cam["cy"]], [0, 0, 1]])
        proj.setImageSize(cam["rows"], cam["cols"])
        cams.append(proj.camera())
    _, conv, corr, lin, prm = gpu_objects(ctx, pairs[0][3])
    prm_c = conv.params()
    prm.outer_iterations, prm.inner_iterations, prm.early_exit_eps = 20, 2, 1e-6
    clouds = [api.Cloud(ctx) for _ in range(2 * npairs)]
    dptrs = [(dev.data_ptr() + int(offs[k]), pairs[k // 2][3]["rows"], pairs[k // 2][3]["cols"])
             for k in range(2 * npairs)]
    fcams = [cams[k // 2] for k in range(2 * npairs)]

    def step(p):
        api.build_batch(ctx, dptrs, fcams, prm_c, clouds, on_device=True)
        return api.align_batch(ctx, clouds[0::2], clouds[1::2], cams, None, corr, lin, p)

    # the autotuner picks launch shapes for this resolution mix on the first
    # (warm-up) call; results do not depend on them
    ctx.set_autotune(True)

    def timed(p):
        for _ in range(warmup):
            step(p)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(steps):
                res = step(p)
            e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, res

    ms, res = timed(prm)
    shape = ctx.launch_shape()
    stats_shape = ctx.stats_shape()
    prm_fixed = L.AlignParams.from_buffer_copy(prm)
    prm_fixed.early_exit_eps = 0.0
    ms_fixed, res_fixed = timed(prm_fixed)
    prof, _ = profile_step(ctx, lambda: step(prm))
    total = sum(v[0] for v in prof.values()) or 1.0
    shares = {k: [round(v[0] / total, 4), v[1]] for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}
    iters = [r.outer_iterations_run for r in res]
    # HBM ceiling of this batch: its algorithmic bytes (two builds and the
    # alignment of every pair, with the iterations each pair ran) at the
    # measured copy bandwidth
    sizes = [c.size() for c in clouds]
    total_bytes = 0.0
    for i, (r, pr) in enumerate(zip(res, pairs)):
        P = pr[3]["rows"] * pr[3]["cols"]
        total_bytes += build_bytes(P, sizes[2 * i]) + build_bytes(P, sizes[2 * i + 1])
        total_bytes += align_bytes(P, sizes[2 * i], r.num_correspondences, r.outer_iterations_run, 2)
    peak, _ = measured_peak_gbs()
    ceiling = npairs / (total_bytes / (peak * 1e9))
    checks = [pose_case(pairs[i][0], pairs[i][1], pairs[i][3], np.array(res[i].T).reshape(4, 4), 20, 2, 1e-6,
                        truth=pairs[i][2]) for i in range(6)]
    errs = [synth.pose_error(np.array(r.T).reshape(4, 4), p[2]) for r, p in zip(res, pairs)]
    ok = [e for e in errs if e[0] < 0.01 and e[1] < 0.02]
    # equal results with and without early exit, where a pair converged
    dT = max(float(np.max(np.abs(np.array(a.T) - np.array(b.T)))) for a, b in zip(res, res_fixed))

    # plain per-pair loop over a sample of the same pairs
    res1 = L.AlignResult()
    pl = []
    for rep in range(2):
        ctx.synchronize()
        t0 = time.perf_counter()
        for i in range(plain_pairs):
            for j in range(2):
                k = 2 * i + j
                ctx.check(ctx.lib.nicp_cloud_from_depth_u16(ctx.h, Cc.c_void_p(dptrs[k][0]), dptrs[k][1], dptrs[k][2],
                                                            0, 1, Cc.byref(cams[i]), Cc.byref(prm_c), None,
                                                            clouds[k].h, None))
            ctx.check(ctx.lib.nicp_align(ctx.h, clouds[2 * i].h, clouds[2 * i + 1].h, Cc.byref(cams[i]), None, None,
                                         None, Cc.byref(corr), Cc.byref(lin), Cc.byref(prm), Cc.byref(res1)))
        ctx.synchronize()
        pl.append(plain_pairs / (time.perf_counter() - t0))
    plain = max(pl)
    value = npairs / (ms / 1e3)
    ctx.set_autotune(False)
    del clouds
    return {"workload": "%d independent pairs, resolutions uniform over %s, offsets 0.5-5 deg / 1-8 cm, "
                        "<= 20 outer x 2 inner, early exit at pose change < 1e-6" % (npairs, "/".join(MIXED_CAMS)),
            "pairs_per_s": value, "ms_per_step": ms, "pairs_per_s_no_early_exit": npairs / (ms_fixed / 1e3),
            "algorithmic_bytes_per_step": total_bytes, "hbm_ceiling_pairs_per_s": ceiling,
            "frac_of_hbm_ceiling": value / ceiling,
            "plain_pairs_per_s": plain, "batched_over_plain": value / plain,
            "outer_iterations_run": {"mean": float(np.mean(iters)), "max": int(max(iters)), "min": int(min(iters))},
            "max_abs_T_diff_vs_no_early_exit": dT,
            "converged_within_0.01rad_2cm": len(ok) / npairs,
            "pose_err_vs_truth_median": {"rad": float(np.median([e[0] for e in errs])),
                                         "m": float(np.median([e[1] for e in errs]))},
            "resolution_counts": {n: names.count(n) for n in MIXED_CAMS},
            "kernel_shares_and_launches": shares, "profiled_step_ms": total,
            "autotuned_launch_shape": {"zbuffer_points_per_thread": shape[0],
                                       "corr_lin_ctas_per_sm": shape[1] or "all that fit",
                                       "stats_threads_x_ctas_per_sm": list(stats_shape),
                                       "resolution_mixes_tuned": shape[2]}}, checks


# ------------------------------------------------------------------ scene fusion leg
def scene_fusion_leg(ctx, seed, frames=30):
    """Frame-to-scene fusion as nicp_aligner.cpp:172-209 maintains its scene:
    every 640x480 frame of the trajectory (Gaussians kept) is added to the
    scene with its pose (Cloud::add) and the scene is merged in that frame's
    view (Merger::merge).  Ground-truth poses; wall time per frame of the
    add + merge calls (both synchronous)."""
    from nicp_b200 import api, synth
    imgs, poses, cam = synth.render_sequence(seed, "640x480", n_frames=frames, period=200)
    proj, conv, _, _, _ = gpu_objects(ctx, cam)
    conv.keepGaussians = True
    clouds = []
    for f in imgs:
        c = api.Cloud(ctx)
        conv.compute(c, f)
        clouds.append(c)
    per_frame = clouds[0].size()
    scene = clouds[0]
    merger = api.Merger(ctx)
    merger.setDepthImageConverter(conv)
    merger.setImageSize(cam["rows"], cam["cols"])
    removed, times = 0, []
    for k in range(1, frames):
        T = synth.rel(poses[0], poses[k]).astype(np.float32)
        ctx.synchronize()
        t0 = time.perf_counter()
        scene.add(clouds[k], T)
        merger.merge(scene, T)
        ctx.synchronize()
        times.append(time.perf_counter() - t0)
        removed += merger.removed
    return {"workload": "%d 640x480 frames fused into one scene (add + merge per frame, ground-truth poses)" % frames,
            "ms_per_frame": 1e3 * float(np.median(times)), "frames_per_s": 1.0 / float(np.median(times)),
            "points_per_frame": per_frame, "scene_points": scene.size(), "removed_points": removed}


# ------------------------------------------------------------------ nearest-neighbour leg
def nn_align_leg(ctx, seed, reps=3):
    """AlignerNN (alignernn.cpp:21-118) on consecutive 640x480 frames of the
    trajectory: exact 6-D nearest-neighbour correspondences every outer
    iteration (10 outer x 1 inner).  Wall time of align() (it synchronises)."""
    from nicp_b200 import api, synth
    imgs, poses, cam = synth.render_sequence(seed, "640x480", n_frames=reps + 1, period=200)
    proj, conv, _, _, _ = gpu_objects(ctx, cam)
    clouds = []
    for f in imgs:
        c = api.Cloud(ctx)
        conv.compute(c, f)
        clouds.append(c)
    al = api.AlignerNN(None, api.Linearizer(ctx), api.CorrespondenceFinderNN(ctx), ctx)
    al.computeStatistics = False
    times, errs = [], []
    for k in range(reps + 1):  # the first pass loads the kernels
        i = min(k, reps - 1)
        al.setReferenceCloud(clouds[i])
        al.setCurrentCloud(clouds[i + 1])
        ctx.synchronize()
        t0 = time.perf_counter()
        T = al.align()
        times.append(time.perf_counter() - t0)
        errs.append(synth.pose_error(T, synth.rel(poses[i], poses[i + 1])))
    return {"workload": "640x480 consecutive frames, exact NN association, 10 outer x 1 inner",
            "ms_per_pair": 1e3 * float(np.median(times[1:])),
            "pose_err_vs_truth_median": {"rad": float(np.median([e[0] for e in errs])),
                                         "m": float(np.median([e[1] for e in errs]))},
            "correspondences": int(al.last_result.num_correspondences)}


# ------------------------------------------------------------------ serving leg
SERVE_MIX = (("320x240", 0.3, 19), ("640x480", 0.6, 38), ("1280x720", 0.1, 7))  # (camera, request share, streams)


def serve_leg(device, rates, seconds, seed, frames_per_stream=16, max_requests=40000, workers=2, submitters=4):
    """Open-loop Poisson load on the serving loop (nicp_server_*): 64 camera
    streams, requests 30/60/10% at 320x240 / 640x480 / 1280x720, each aligned
    against its stream's device-resident keyframe (replaced when inliers fall
    below 40% of its points), admission against a 60 GB budget.  A stream
    replays a 16-frame stretch of a 200-frame loop back and forth, so
    consecutive requests of a stream are one trajectory step apart.  Latency
    is submit -> result published, measured inside the server."""
    from concurrent.futures import ThreadPoolExecutor
    from nicp_b200 import _lib as L
    from nicp_b200 import api, synth

    streams = []  # (camera name, frames, poses, Camera)
    jobs = []
    for name, _, count in SERVE_MIX:
        for _ in range(count):
            jobs.append((seed + 31 * len(jobs), name))
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        rendered = list(ex.map(lambda j: synth.render_sequence(j[0], j[1], n_frames=frames_per_stream, period=200),
                               jobs))
    for (sd, name), (frames, poses, cam) in zip(jobs, rendered):
        c = L.Camera()
        L.load().nicp_default_camera(c)
        c.fx, c.fy, c.cx, c.cy = cam["fx"], cam["fy"], cam["cx"], cam["cy"]
        c.rows, c.cols = cam["rows"], cam["cols"]
        streams.append((name, [np.ascontiguousarray(f) for f in frames], poses, c, cam))
    by_cam, base = [], 0
    for name, share, count in SERVE_MIX:
        by_cam.append(list(range(base, base + count)))
        base += count
    shares = np.array([s for _, s, _ in SERVE_MIX])

    def frame_of(k):  # back-and-forth replay: 0..15..1, 0..15..1, ...
        p = 2 * (frames_per_stream - 1)
        k %= p
        return k if k < frames_per_stream else p - k

    srv = api.Server(device=device, hbm_budget_bytes=60 << 30, max_batch=64, workers=workers)
    seq = [0] * len(streams)
    rid = [0]

    def submit(s, t_sub, meta):
        k = seq[s]
        seq[s] += 1
        i = rid[0]
        rid[0] += 1
        meta[i] = (s, frame_of(k))
        t_sub[i] = time.perf_counter()
        srv.submit(s, i, streams[s][1][frame_of(k)], streams[s][3])

    # warm-up: a burst of 3 requests per stream (sizes the pools and
    # workspaces, sets every stream's keyframe), then a settle
    out = []
    samples = []  # served requests checked against the FP64 oracle (CPU leg)
    track = {}  # per stream: (keyframe frame, last two estimates against it), in request order

    def follow(results, meta):
        """Advances the per-stream keyframe tracking through a phase's results."""
        for r in sorted(results, key=lambda r: r["request_id"]):
            if r["status"] != 0:
                continue
            key, hist = track.get(r["stream_id"], (None, []))
            f = meta[r["request_id"]][1]
            if r["keyframe_replaced"]:
                key, hist = f, []
            elif key is not None:
                hist = (hist + [np.asarray(r["T"], float).reshape(4, 4)])[-2:]
            track[r["stream_id"]] = (key, hist)

    wmeta, wt = {}, {}
    for _ in range(3):
        for s in range(len(streams)):
            submit(s, wt, wmeta)
    follow(srv.drain(len(wmeta), timeout_s=300), wmeta)
    # unmeasured Poisson phases first: 1 s at 2000 requests/s (every worker
    # meets every resolution: pools, first launches), then 1 s at 10000
    # requests/s (batches reach max size: workspaces and pools grow to their
    # steady-state sizes before any measured rate)
    warm = [(2000.0, 1.0, False), (10000.0, 1.0, False)]
    for rate, window, measured in warm + [(r, seconds, True) for r in rates]:
        rng = np.random.default_rng(seed + int(rate) + (0 if measured else 7))
        n = int(min(max_requests, rate * window))
        cams = rng.choice(len(SERVE_MIX), size=n, p=shares)
        sid = np.array([by_cam[c][rng.integers(len(by_cam[c]))] for c in cams])
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
        meta, t_sub = {}, {}
        first = rid[0]
        # submitters: streams are split between threads (a stream's requests
        # stay in order); each follows the arrival times of its streams
        lock = threading.Lock()

        def run(t, t0):
            mine = np.nonzero(sid % submitters == t)[0]
            for i in mine:
                due = t0 + arrivals[i]
                while time.perf_counter() < due:
                    pass
                with lock:
                    k = seq[sid[i]]
                    seq[sid[i]] += 1
                    j = first + int(i)
                meta[j] = (int(sid[i]), frame_of(k))
                t_sub[j] = time.perf_counter()
                srv.submit(int(sid[i]), j, streams[sid[i]][1][frame_of(k)], streams[sid[i]][3])

        t0 = time.perf_counter() + 0.01
        th = [threading.Thread(target=run, args=(t, t0)) for t in range(submitters)]
        for x in th:
            x.start()
        results = []
        while any(x.is_alive() for x in th):
            results += srv.poll(wait_ms=5)
        for x in th:
            x.join()
        t_submitted = max(t_sub.values())
        rid[0] = first + n
        results += srv.drain(n - len(results), timeout_s=300)
        ok = [r for r in results if r["status"] == 0]
        lat = np.array([r["latency_ms"] for r in ok])
        q = np.array([r["queue_ms"] for r in ok])
        end = max(t_sub[r["request_id"]] + r["latency_ms"] / 1e3 for r in ok) if ok else t_submitted
        # pose error vs ground truth: replay each stream's results in order
        # (the keyframe of a stream's first request here is the one the
        # previous load left: unknown frame, so that request is skipped)
        errs, replaced = [], 0
        per_stream = {}
        for r in sorted(ok, key=lambda r: r["request_id"]):
            per_stream.setdefault(r["stream_id"], []).append(r)
        for s, rs in per_stream.items():
            # the stream's keyframe and estimates carry over from the earlier
            # phases (every phase drains before the next starts)
            key, hist = track.get(s, (None, []))
            poses = streams[s][2]
            for r in rs:
                f = meta[r["request_id"]][1]
                if key is not None:  # T maps the frame into the keyframe it was aligned against
                    errs.append(synth.pose_error(r["T"], synth.rel(poses[key], poses[f])))
                    # the server's guess: constant velocity over the last two estimates
                    g = np.eye(4) if not hist else hist[-1] if len(hist) < 2 else \
                        hist[-1] @ np.linalg.inv(hist[-2]) @ hist[-1]
                    name = streams[s][0]
                    if measured and len(samples) < 6 and sum(c["cam"]["cols"] == streams[s][4]["cols"]
                                                             for c in samples) < 2:
                        samples.append(pose_case(streams[s][1][key], streams[s][1][f], streams[s][4], r["T"],
                                                 guess=g, truth=synth.rel(poses[key], poses[f])))
                if r["keyframe_replaced"]:
                    key, hist = f, []
                    replaced += 1
                elif key is not None:
                    hist = (hist + [np.asarray(r["T"], float).reshape(4, 4)])[-2:]
            track[s] = (key, hist)
        er = np.array([e[0] for e in errs]) if errs else np.zeros(1)
        et = np.array([e[1] for e in errs]) if errs else np.zeros(1)
        if not measured:
            while srv.status()[0]:
                time.sleep(0.01)
            continue
        out.append({"offered_rps": rate, "submitted_rps": n / (t_submitted - t0), "requests": n,
                    "completed": len(ok), "failed": len(results) - len(ok), "lost": n - len(results),
                    "throughput_rps": len(ok) / (end - t0),
                    "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
                    "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
                    "queue_p50_ms": float(np.percentile(q, 50)) if len(q) else None,
                    "mean_batch": float(np.mean([r["batch_size"] for r in ok])) if ok else None,
                    "keyframe_replacements": replaced,
                    "pose_err_vs_truth": {"rad_p50": float(np.median(er)), "rad_p99": float(np.percentile(er, 99)),
                                          "m_p50": float(np.median(et)), "m_p99": float(np.percentile(et, 99))}})
        # let the queue empty before the next rate
        while srv.status()[0]:
            time.sleep(0.01)
    srv.close()
    return {"streams": len(streams), "mix": {n: s for n, s, _ in SERVE_MIX}, "budget_gb": 60, "workers": workers,
            "max_batch": 64, "submitter_threads": submitters, "arrivals": "poisson, open loop",
            "seconds_per_rate": seconds,
            "warmup": "3 requests per stream (burst), then 1 s of Poisson arrivals at 2000 and 1 s at 10000 requests/s", "rates": out}, samples


def workload_config(args):
    return {"workload": "640x480 frame-to-frame sequence, %d frames (%d pairs), reference defaults, "
                        "%d outer x 1 inner" % (args.frames, args.frames - 1, 10),
            "resolution": "640x480", "frames": args.frames, "pairs_per_step": args.frames - 1,
            "camera": "fx=fy=525 cx=319.5 cy=239.5", "moments": "fp64", "cross_block": "fp64",
            "solve": "fp64 ldlt on device", "statistics": "not computed (optional post-pass)",
            "l2": "inputs larger than L2 (clouds ~4.9 GB per step)", "parallelism": "replicas",
            "launch_shapes": "default" if getattr(args, "no_autotune", False) else
                             "autotuned per resolution during warm-up (bitwise the default's results)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--frames", type=int, default=200)
    ap.add_argument("--period", type=int, default=None,
                    help="trajectory loop length in frames (default: --frames); a short run with --period 200 "
                         "has the per-frame motion of the 200-frame workload (small profiling cases)")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--oracle-pairs", type=int, default=10,
                    help="pairs of the timed sequence checked against the FP64 oracle (CPU leg)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain one-pair-per-call leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop leg")
    ap.add_argument("--no-mixed", action="store_true", help="skip the 512-pair mixed-resolution batch leg")
    ap.add_argument("--no-fusion", action="store_true", help="skip the scene-fusion (merger) leg")
    ap.add_argument("--no-nn", action="store_true", help="skip the nearest-neighbour aligner leg")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default launch shapes in the headline legs (otherwise tuned per resolution during warm-up; "
                         "results are bitwise the same)")
    ap.add_argument("--serve-rates", default="500,2000,5000,10000,20000",
                    help="Poisson arrival rates (requests/s) of the serving leg")
    ap.add_argument("--serve-seconds", type=float, default=1.5, help="arrival window per rate")
    ap.add_argument("--serve-workers", type=int, default=4, help="server worker threads (one context each)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", timeout=timedelta(seconds=600))

    if args.impl == "reference":
        rc = reference_arm(args, rank, world)
        if dist:
            dist.destroy_process_group()
        return rc

    import torch
    from nicp_b200 import api

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)
    ctx = api.Context(local, stream.cuda_stream)
    frames, poses, cam = make_workload(args.seed + 7919 * rank, args.frames, period=args.period)
    F = len(frames)
    npairs = F - 1
    proj, conv, corr, lin, prm = gpu_objects(ctx, cam)
    cam_c = proj.camera(cam["rows"], cam["cols"])
    prm_c = conv.params()
    clouds = [api.Cloud(ctx) for _ in range(F)]

    # device-resident inputs
    dev = torch.from_numpy(frames.astype(np.int16, copy=False).view(np.int16)).to(f"cuda:{local}")
    P = cam["rows"] * cam["cols"]
    dptrs = [(dev.data_ptr() + 2 * P * i, cam["rows"], cam["cols"]) for i in range(F)]
    host = torch.from_numpy(frames.view(np.int16)).pin_memory()
    hframes = [host[i].numpy().view(np.uint16) for i in range(F)]

    def step_dev():
        return run_step(ctx, dptrs, cam_c, prm_c, clouds, corr, lin, prm, True)

    def step_host():
        return run_step(ctx, hframes, cam_c, prm_c, clouds, corr, lin, prm, False)

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        return max_over_ranks_of(dist, x)

    # the clock sampler starts before the warm-up: nvidia-smi's start-up is
    # not inside the timed region
    clocks = ClockSampler(local)
    clocks.start()
    # the first warm-up step tunes the launch shapes of this resolution
    # (build: stats kernel shape; alignment: z-buffer points per thread,
    # fused-kernel CTAs per SM); every shape gives bitwise the same clouds
    # and poses
    ctx.set_autotune(not args.no_autotune)
    for _ in range(args.warmup):
        step_dev()
    torch.cuda.synchronize()
    zb_ppt, corr_ctas, _ = ctx.launch_shape()
    st_thr, st_ctas = ctx.stats_shape()
    headline_shape = {"zbuffer_points_per_thread": zb_ppt, "corr_lin_ctas_per_sm": corr_ctas or "all that fit",
                      "stats_threads_x_ctas_per_sm": [st_thr, st_ctas]}

    # ---- value: device-resident inputs
    l0 = ctx.kernel_launches()
    barrier()
    torch.cuda.synchronize()
    clocks.mark(0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            res = step_dev()
        e1.record(stream)
    torch.cuda.synchronize()
    clocks.mark(1)
    barrier()
    launches = ctx.kernel_launches() - l0
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    ms = max_over_ranks(ms)
    value = replica_value(world, npairs, args.steps, ms)

    # ---- e2e: pinned host frames through the C ABI, results back to the host
    for _ in range(2):
        step_host()
    h0, d0 = ctx.transfer_bytes()
    barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e2.record(stream)
        for _ in range(args.steps):
            step_host()
        e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    h1, d1 = ctx.transfer_bytes()
    ms_e2e = max_over_ranks(e2.elapsed_time(e3))
    e2e = replica_value(world, npairs, args.steps, ms_e2e)

    # ---- accuracy against the synthetic ground truth (median over pairs)
    from nicp_b200 import synth
    errs = [synth.pose_error(np.array(r.T).reshape(4, 4), synth.rel(poses[i], poses[i + 1]))
            for i, r in enumerate(res)]
    rot_med = float(np.median([e[0] for e in errs]))
    tr_med = float(np.median([e[1] for e in errs]))

    # ---- per-kernel shares and the roofline of the top kernel
    prof, res_p = profile_step(ctx, step_dev)
    total = sum(v[0] for v in prof.values()) or 1.0
    top = max(prof, key=lambda k: prof[k][0])
    Vs = [c.size() for c in clouds[:4]]
    V = float(np.mean(Vs))
    C = float(np.mean([r.num_correspondences for r in res_p]))  # accepted; candidates are >= this
    peak, peak_kind = measured_peak_gbs()
    top_ms, top_n = prof[top]
    launches_per_step = top_n
    per_launch_bytes = {
        "corr_lin": (20 * P + 56 * C) * npairs,
        "zbuffer": (16 * V + 8 * V) * npairs,
        "stats_omega": (10 * 8 * P + 6 * P + 28 * V) * F,  # implicit Omega
        "moments_bands": (2 * P + 3 * 80 * P / 16) * F / 2,  # two kernels per stage launch
        "moments_sweep": (2 * P + 80 * P / 16 + 80 * P) * F,
        "unproject": (2 * P + 4 * P + 12 * V) * F / 2,  # two kernels per stage launch
        "resolve": (20 * P) * npairs,  # z-buffer read 8P, index write 4P, z-buffer reset 8P
    }.get(top, 0.0)
    achieved = per_launch_bytes / (top_ms / top_n / 1e3) / 1e9
    roof = {"kernel": top, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": measured_traffic(top, {"pair": npairs, "frame": F}),
            "traffic_source": "profiles/dram_traffic_640x480_seq.txt (ncu, 19-pair case scaled per pair/frame)",
            "bytes_per_launch": per_launch_bytes, "avg_launch_ms": top_ms / top_n,
            "shares": {k: round(v[0] / total, 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}}

    # ---- plain one-pair-per-call path
    plain = None
    if not args.no_plain and rank == 0:
        from nicp_b200 import _lib as L
        import ctypes as Cc
        pl = []
        prm1 = L.AlignParams()
        ctx.lib.nicp_default_align_params(prm1)
        prm1.compute_statistics = 0
        res1 = L.AlignResult()
        nplain = min(npairs, 60)
        for rep in range(2):
            ctx.synchronize()
            t0 = time.perf_counter()
            ctx.check(ctx.lib.nicp_cloud_from_depth_u16(ctx.h, Cc.c_void_p(dptrs[0][0]), cam["rows"], cam["cols"], 0,
                                                        1, Cc.byref(cam_c), Cc.byref(prm_c), None, clouds[0].h, None))
            for i in range(nplain):
                ctx.check(ctx.lib.nicp_cloud_from_depth_u16(ctx.h, Cc.c_void_p(dptrs[i + 1][0]), cam["rows"],
                                                            cam["cols"], 0, 1, Cc.byref(cam_c), Cc.byref(prm_c), None,
                                                            clouds[i + 1].h, None))
                ctx.check(ctx.lib.nicp_align(ctx.h, clouds[i].h, clouds[i + 1].h, Cc.byref(cam_c), None, None, None,
                                             Cc.byref(corr), Cc.byref(lin), Cc.byref(prm1), Cc.byref(res1)))
            ctx.synchronize()
            pl.append(nplain / (time.perf_counter() - t0))
        plain = max(pl)

    # whole step: every frame built once, every pair aligned (10 outer x 1 inner)
    step_bytes = F * build_bytes(P, V) + npairs * align_bytes(P, V, C, 10, 1)
    whole_step = {"algorithmic_bytes": step_bytes, "gbs": step_bytes / (ms / args.steps / 1e3) / 1e9,
                  "frac": step_bytes / (ms / args.steps / 1e3) / 1e9 / peak,
                  "hbm_ceiling_pairs_per_s": npairs / (step_bytes / (peak * 1e9))}

    mixed, mixed_checks = None, []
    if not args.no_mixed and rank == 0:
        mixed, mixed_checks = mixed_batch_leg(ctx, stream, local, args.seed + 17)

    fusion = None
    if not args.no_fusion and rank == 0:
        fusion = scene_fusion_leg(ctx, args.seed + 29)

    nn = None
    if not args.no_nn and rank == 0:
        nn = nn_align_leg(ctx, args.seed + 41)

    serving, serve_checks = None, []
    if not args.no_serve and rank == 0:
        serving, serve_checks = serve_leg(local, [float(r) for r in args.serve_rates.split(",")], args.serve_seconds,
                                          args.seed, workers=args.serve_workers)

    cpu, oracle_seq, oracle_mixed, oracle_served = None, None, None, None
    if not args.no_cpu and rank == 0:
        v, n, dt, threads = cpu_baseline(frames, cam, seconds=args.cpu_seconds)
        cpu = {"value": v, "unit": "pairs/s", "cores": threads, "kind": "port",
               "sample": "%d consecutive 640x480 frame pairs (build + align, oracle REF32, %d threads, %.1f s)"
                         % (n, threads, dt)}
        # the checker: the first pairs of the timed workload (and a few
        # mixed-batch pairs) against the oracle's FP64 pipeline
        seq_cases = [pose_case(frames[i], frames[i + 1], cam, np.array(res[i].T).reshape(4, 4),
                               truth=synth.rel(poses[i], poses[i + 1]))
                     for i in range(min(args.oracle_pairs, npairs))]
        oracle_seq = oracle_pose_check(seq_cases, threads)
        oracle_mixed = oracle_pose_check(mixed_checks, threads) if mixed_checks else None
        oracle_served = oracle_pose_check(serve_checks, threads) if serve_checks else None

    if rank == 0:
        # the headline figures first (scalars), the bulky per-leg records last
        rates = (serving or {}).get("rates", [])
        summary = {
            "plain_pairs_per_s": plain, "batched_over_plain": (value / world / plain) if plain else None,
            "pose_err_vs_oracle_rad_max": oracle_seq["rad_max"] if oracle_seq else None,
            "pose_err_vs_oracle_m_max": oracle_seq["m_max"] if oracle_seq else None,
            "pose_err_vs_oracle_pairs": oracle_seq["pairs"] if oracle_seq else None,
            "whole_step_gbs": whole_step["gbs"], "whole_step_frac": whole_step["frac"],
            "hbm_ceiling_pairs_per_s": whole_step["hbm_ceiling_pairs_per_s"],
            "mixed_pairs_per_s": mixed["pairs_per_s"] if mixed else None,
            "mixed_plain_pairs_per_s": mixed["plain_pairs_per_s"] if mixed else None,
            "mixed_batched_over_plain": mixed["batched_over_plain"] if mixed else None,
            "mixed_frac_of_hbm_ceiling": mixed["frac_of_hbm_ceiling"] if mixed else None,
            "mixed_pose_err_vs_oracle_rad_max": oracle_mixed["rad_max"] if oracle_mixed else None,
            "mixed_pairs_diverged_in_fp64": len(oracle_mixed["diverged"]) if oracle_mixed else None,
            "served_pose_err_vs_oracle_rad_max": oracle_served["rad_max"] if oracle_served else None,
        }
        for r in rates:
            summary["serve_%d_rps_p50_ms" % r["offered_rps"]] = r["p50_ms"]
            summary["serve_%d_rps_p99_ms" % r["offered_rps"]] = r["p99_ms"]
            summary["serve_%d_rps_throughput" % r["offered_rps"]] = r["throughput_rps"]
        line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(args),
                "roofline": roof, "cpu_baseline": cpu,
                "e2e": {"value": e2e, "unit": "pairs/s", "h2d_bytes_per_step": (h1 - h0) // args.steps,
                        "d2h_bytes_per_step": (d1 - d0) // args.steps},
                "gpu_launches": int(launches), "clocks": clk}
        line["config"]["launch_shape"] = headline_shape
        line.update(summary)
        line.update({"pose_err_vs_truth_median": {"rad": rot_med, "m": tr_med},
                     "pose_err_vs_oracle": {"sequence": oracle_seq, "mixed_batch": oracle_mixed,
                                            "served": oracle_served},
                     "whole_step": whole_step, "points_per_frame": V, "correspondences_per_pair": C,
                     "mixed_batch": mixed, "scene_fusion": fusion, "nn_align": nn, "serving": serving})
        print(json.dumps(line), flush=True)
    del clouds
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
