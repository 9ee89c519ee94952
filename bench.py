"""GPIS path samples/s on B200: the configuration-0 render.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one full render of the configuration-0 scene: 256x256 pixels x 20
passes (1,310,720 path samples; sphere mean (0,0,-500) r=70 in a null sphere
r=130, renewal_plus, SE kernel sigma 1 / length 1 / aniso (1,1,1), 3 points per
cell, max_bounce 10, constant sky 1.0). Under torchrun every rank renders its
own 20 passes (pass offset rank*20: weak scaling) and the framebuffers are
summed with one all_reduce per step. Path state (~220 MB) exceeds the 126 MB L2
and a 256 MB buffer is written between steps as well.

`--impl reference` times the reference's own CPU implementation
(oracle/_ref/libmupsi_ref_timing.so: its sources at -O3 with OpenMP; the C
restatement of the oracle when that library is absent) with every host
thread: each step traces a different seeded random subset of the scene's
pixels (disjoint subsets) at all 20 passes, and the value is the samples of the
timed steps over their time (the per-step median is reported beside it).

The default run also measures configurations 1-4 (`extras`), each with a CPU
baseline from the same reference build on a bounded sample of that workload
and a roofline fraction, and the configuration-0 image in expectation
(`image_parity`: per-pixel 3-sigma band against the reference's samples and
image RMSE against a 4096-spp FP64-accumulated render).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GPIS path samples/s (configuration-0 render)"
UNIT = "samples/s"
W, H, SPP = 256, 256, 20
SAMPLES_PER_STEP = W * H * SPP


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=3.0, help="CPU work per reference step")
    ap.add_argument("--extras", type=int, default=1, help="also time configurations 1-4 (single GPU)")
    ap.add_argument("--parity", type=int, default=1, help="also compare the configuration-0 image in expectation")
    ap.add_argument("--only", choices=EXTRAS, default=None,
                    help="time only this configuration (its JSON object, no bench line)")
    return ap.parse_args()


def _config(extra=None):
    c = {"workload": "config0: sphere-mean GPIS render 256x256x20spp, renewal_plus, sigma 1, length 1, "
                     "aniso (1,1,1), 3 pts/cell, max_bounce 10, constant sky",
         "width": W, "height": H, "spp": SPP, "max_bounce": 10, "l2": "state > L2 (126 MB) and 256 MB flush "
                                                                       "between steps"}
    if extra:
        c.update(extra)
    return c


# ------------------------------------------------------------------ CPU side
def _cpu_info():
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count()


def _cpu_engine():
    from oracle import bind
    if bind.ref_available("ref_timing"):
        return "reference", bind.RefOracle("ref_timing")
    return "port", bind.PortOracle()


class _StdoutToStderr:
    """The reference's loader prints progress on stdout (file descriptor 1);
    the bench's stdout carries only its JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def _cpu_scene_load(engine_kind, engine, scene, name):
    """The scene in the CPU engine: the reference through its own scene.json
    loader (Controller::load), the restatement from the descriptor."""
    if engine_kind == "reference":
        with _StdoutToStderr():
            return _reference_scene(engine, scene, tempfile.mkdtemp(), name)
    return engine.scene_create(scene.desc())


def _pixel_subsets(w, h, npix, count, seed):
    """`count` disjoint seeded random subsets of npix pixels each."""
    perm = np.random.default_rng(seed).permutation(w * h)
    npix = max(1, min(npix, (w * h) // count))
    return [perm[i * npix:(i + 1) * npix] for i in range(count)]


def _samples(pix, w, passes, k0=0):
    xs = np.repeat(pix % w, passes).astype(np.int32)
    ys = np.repeat(pix // w, passes).astype(np.int32)
    ks = np.tile(np.arange(k0, k0 + passes, dtype=np.int32), len(pix))
    return xs, ys, ks


def cpu_render_rate(eng, h, w, hh, passes, seconds, subsets, k0=0, seed=0, keep=False, warmup=0):
    """Time PathTracer::trace on `subsets` disjoint random pixel subsets of the
    image, every pixel at passes [k0, k0 + passes), sized together to about
    `seconds`. Returns the rate over all timed subsets, the per-subset rates and
    (keep) the traced pixels and radiance."""
    # the rate from a probe of random pixels (one pass each), grown until it
    # takes a measurable time
    rate0, m = 0.0, 16
    for _ in range(8):
        probe = _pixel_subsets(w, hh, m, 1, seed + 1000)[0]
        t = time.perf_counter()
        eng.trace(h, *_samples(probe, w, 1, k0))
        dt = time.perf_counter() - t
        rate0 = len(probe) / max(1e-6, dt)
        if dt > 0.05 * seconds or len(probe) >= w * hh:
            break
        m *= 4
    npix = int(max(4, rate0 * seconds / max(1, subsets + warmup) / passes))
    subs = _pixel_subsets(w, hh, npix, subsets + warmup, seed)
    rates, n_all, t_all, kept = [], 0, 0.0, []
    for i, pix in enumerate(subs):
        xs, ys, ks = _samples(pix, w, passes, k0)
        t = time.perf_counter()
        rad = eng.trace(h, xs, ys, ks)
        dt = time.perf_counter() - t
        if i < warmup:
            continue
        rates.append(len(xs) / dt)
        n_all += len(xs)
        t_all += dt
        if keep:
            kept.append((pix, rad.reshape(len(pix), passes, 3)))
    out = {"value": n_all / t_all, "median": float(np.median(rates)), "min": float(min(rates)),
           "max": float(max(rates)), "subsets": len(rates), "pixels_per_subset": len(subs[-1]),
           "samples": n_all, "seconds": t_all}
    if keep:
        out["kept"] = kept
    return out


def _cpu_desc(kind, eng, r, what):
    model, cores = _cpu_info()
    threads = eng.num_threads() if kind == "reference" else cores
    return threads, (f"{what}: {r['subsets']} disjoint seeded random subsets of {r['pixels_per_subset']} pixels, "
                     f"{r['samples']} path samples in {r['seconds']:.1f} s (per-subset rates {r['min']:.0f}-"
                     f"{r['max']:.0f}, median {r['median']:.0f} samples/s), {threads} OpenMP threads on {model}")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from mupsi_b200 import scene as S
    kind, eng = _cpu_engine()
    sc = S.config0_scene(W, H, SPP)
    h = _cpu_scene_load(kind, eng, sc, "config0")
    r = cpu_render_rate(eng, h, W, H, SPP, args.cpu_seconds * (args.steps + args.warmup), args.steps,
                        warmup=args.warmup, seed=7)
    threads, sample = _cpu_desc(kind, eng, r, "each step one subset of the configuration-0 image at all 20 passes")
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * r["seconds"] / r["subsets"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": _config({"parallelism": "openmp", "sample": sample}),
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": threads, "kind": kind, "sample": sample,
                             "median_of_steps": r["median"]},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU side
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device_index), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        rows = [[c.strip() for c in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows)}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


# Source-level operations per impulse evaluation of the march's psi sum (the
# roofline unit): 4 PCG32 steps at 10 integer ops each (64-bit multiply-add as
# three 32-bit multiply-adds plus carry, xorshift, rotate), 3 mantissa-trick
# uniforms for the position (shift/or, subtract: 1 integer + 1 float each), the
# weight's sign bit put onto the Gaussian (1 three-input logic op), the impulse
# position (3 multiply + 3 add), |p - s|^2 (3 sub, 1 mul, 2 fused multiply-add),
# the exponent scale (1 mul), exp2 on the SFU (1), the signed accumulate (1 add):
# 44 integer + 18 float = 62 issue slots, 1 of them on the SFU.
OPS_PER_IMPULSE = 62
# the gradient adds (w h) c2 (1 multiply) and three multiply + add pairs
OPS_PER_IMPULSE_GRAD = 69
BVH_NODE_BYTES, BVH_TRI_BYTES = 32, 48  # node; leaf-ordered triangle record (3 vertices + id, padded)


def issue_bound(ops, local=0):
    """Impulse evaluations/s the SMs can issue at `ops` operations each
    (4 schedulers x 32 lanes per SM, one instruction per clock, measured max clock)."""
    import torch
    peaks, kind = _peaks()
    mhz = float(peaks.get("sm_max_mhz", 1965.0))
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    return sms * 4 * 32 * mhz * 1e6 / ops, f"{sms} SMs x 128 lanes x {mhz:.0f} MHz ({kind} sm_max_mhz) / {ops} ops"


def l2_bandwidth():
    """Measured L2 bandwidth: a CUDA graph of 64 copies between two 24 MB
    buffers (both resident in the 126 MB L2), read + write bytes per second."""
    import torch
    a = torch.ones(6 << 20, dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    for _ in range(3):
        b.copy_(a)
    g = torch.cuda.CUDAGraph()
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        with torch.cuda.graph(g, stream=st):
            for i in range(64):
                (b if i % 2 == 0 else a).copy_(a if i % 2 == 0 else b)
    torch.cuda.synchronize()
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del g
    return 64 * 2 * a.numel() * 4 / (best / 1e3) / 1e9


def march_roofline(st, samples, ops=OPS_PER_IMPULSE, bvh=None, l2_gbs=None, hbm_gbs=None):
    """Roofline figures of a render's march kernels from its profile stats:
    impulse evaluations/s against the issue bound and, for mesh means, the BVH
    algorithmic bytes/s (nodes x 32 + triangles x 52, from a counted render of
    the same work, `bvh` = (bytes per sample)) against measured L2 and HBM."""
    peak, basis = issue_bound(ops)
    ms = st["march_ms"]
    achieved = st["impulse_evals"] / (ms / 1e3) if ms > 0 else 0.0
    out = {"bound": "issue", "kernel": "k_march", "achieved": achieved / 1e9, "peak": peak / 1e9,
           "unit": "Gimpulse-evals/s", "frac": achieved / peak, "peak_basis": basis,
           "march_ms": ms, "march_share": ms / max(1e-9, ms + st["shade_ms"]),
           "psi_evals_per_sample": st["psi_evals"] / samples, "march_steps_per_sample": st["march_steps"] / samples}
    if bvh is not None:
        gbs = bvh * samples / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        out["bvh"] = {"bytes_per_sample": bvh, "achieved_gbs": gbs, "l2_gbs": l2_gbs, "hbm_gbs": hbm_gbs,
                      "frac_l2": gbs / l2_gbs if l2_gbs else None, "frac_hbm": gbs / hbm_gbs if hbm_gbs else None,
                      "basis": "(nodes loaded x 32 B + triangles tested x 48 B) of the marches' and shading's "
                               "BVH queries, counted on the device, / march kernel time"}
        out["mean_evals_per_sample"] = st["mean_evals"] / samples
    return out


def march_per_iteration(sc, st, pass0, pass1, fb, flush):
    """The march roofline per bounce iteration of a render: each iteration's
    impulse evaluations are the difference of two renders whose max_bounce
    differs by one (iteration i runs the same marches in every render that
    reaches it), set against that iteration's march time in the profiled
    full render `st`."""
    from mupsi_b200 import scene as S
    from mupsi_b200.api import GpuRenderer, GpuScene
    peak, _ = issue_bound(OPS_PER_IMPULSE)
    imps = [0]
    for b in range(1, sc.max_bounce + 1):
        sb = S.config0_scene(sc.width, sc.height, sc.spp)
        sb.max_bounce = b
        g = GpuScene(sb)
        r = GpuRenderer()
        r.prepare_render(g)
        g.profile(True)
        flush.fill_(4)
        r.start_render_progressive(pass1, spp_begin=pass0, out=fb)
        imps.append(g.stats(reset=True)["impulse_evals"])
        g.close()
    rows = []
    for i in range(sc.max_bounce):
        ms = float(st["iter_march_ms"][i])
        n = imps[i + 1] - imps[i]
        rate = n / (ms / 1e3) if ms > 0 else 0.0
        rows.append({"iteration": i, "rays": int(st["iter_medium"][i]), "impulse_evals": int(n),
                     "march_ms": round(ms, 4), "Gimpulse_evals_s": round(rate / 1e9, 2),
                     "frac": round(rate / peak, 4)})
    return rows


def bvh_bytes_per_sample(gs, render, samples):
    """Algorithmic BVH bytes per path sample of `render()` (counted traversals)."""
    gs.profile(True, bvh=True)
    gs.stats(reset=True)
    render()
    st = gs.stats(reset=True)
    gs.profile(False)
    return (st["bvh_nodes"] * BVH_NODE_BYTES + st["bvh_tris"] * BVH_TRI_BYTES) / samples, st


def run_gpu(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from mupsi_b200 import scene as S
    from mupsi_b200.api import GpuRenderer, GpuScene
    from mupsi_b200.lib import launch_count

    stream = torch.cuda.current_stream()
    sc = S.config0_scene(W, H, SPP)
    gs = GpuScene(sc)
    rend = GpuRenderer()
    rend.prepare_render(gs)
    from mupsi_b200.multigpu import combine, pass_range
    fb = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # weak scaling: SPP passes per rank, SPP * world passes in the whole image
    pass0, pass1 = pass_range(SPP * world, world, rank)

    def step():
        rend.start_render_progressive(pass1, spp_begin=pass0, out=fb)
        if world > 1:
            combine(fb, pass1 - pass0, SPP * world)

    for _ in range(args.warmup):
        flush.fill_(1)
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local) if rank == 0 else None
    time.sleep(0.3)
    l0 = launch_count()
    total_ms = 0.0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    for _ in range(args.steps):
        flush.fill_(2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    launches = launch_count() - l0
    time.sleep(0.2)
    clk = clocks.stop() if clocks else None
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_per_step = t.item() / args.steps
    value = SAMPLES_PER_STEP * world / (ms_per_step / 1000.0)

    # roofline of the dominant kernel (the march), timed live with CUDA events
    gs.profile(True)
    gs.stats(reset=True)
    for _ in range(2):
        flush.fill_(3)
        rend.start_render_progressive(pass1, spp_begin=pass0, out=fb)
    st = gs.stats(reset=True)
    gs.profile(False)
    roof = march_roofline(st, 2.0 * SAMPLES_PER_STEP)
    roof.update({"traffic": None,
                 "traffic_note": "not measurable inside the run (no device counters without a profiler); "
                                 "ncu's DRAM bytes for this kernel are in profiles/",
                 "launches": st["march_launches"], "ms_per_launch": st["march_ms"] / max(1, st["march_launches"]),
                 "impulse_evals_per_launch": st["impulse_evals"] / max(1, st["march_launches"]),
                 "iter_rays": st["iter_medium"][:10], "iter_march_ms": [round(x, 4) for x in st["iter_march_ms"][:10]]})
    if world == 1:
        roof["per_iteration"] = march_per_iteration(sc, st, pass0, pass1, fb, flush)

    # end to end through the public API with pinned host buffers: scene upload,
    # render, framebuffer read back, release, every step
    host_fb = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True).numpy()
    e2e_times = []
    e2e_parts = []
    desc_bytes = 0
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g2 = GpuScene(sc)
        r2 = GpuRenderer()
        r2.prepare_render(g2)
        t1 = time.perf_counter()
        r2.start_render_progressive(pass1, spp_begin=pass0, out=host_fb)
        t2 = time.perf_counter()
        g2.close()
        if i >= args.warmup:
            e2e_times.append(time.perf_counter() - t0)
            e2e_parts.append((t1 - t0, t2 - t1, time.perf_counter() - t2))
    # bytes the scene create copies host->device: descriptor + march table (4001 floats)
    desc_bytes = 4 * 4001 + 8192
    e2e_t = torch.tensor([sum(e2e_times)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_val = SAMPLES_PER_STEP * world * len(e2e_times) / e2e_t.item()

    extras = run_extras(args) if (rank == 0 and world == 1 and args.extras) else None

    cpu = parity = None
    if rank == 0 and world == 1:
        cpu, kept = cpu_baseline_config0(sc, seconds=15.0)
        parity = image_parity_config0(gs, kept) if args.parity else None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": _config({"parallelism": f"spp-sharded x{world}" if world > 1 else "single GPU",
                                   "global_batch": SAMPLES_PER_STEP * world}),
                "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": desc_bytes,
                        "d2h_bytes_per_step": W * H * 3 * 4,
                        "step_ms": [round(1e3 * t, 3) for t in e2e_times],
                        "median_create_render_destroy_ms": [round(1e3 * float(np.median([p[k] for p in e2e_parts])), 3)
                                                            for k in range(3)]},
                "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clk}
        if parity:
            line["image_parity"] = parity
        if extras:
            line["extras"] = extras
        print(json.dumps(line), flush=True)
    gs.close()
    if world > 1:
        dist.destroy_process_group()


def cpu_baseline_config0(sc, seconds):
    """The reference's timing build on 5 disjoint random pixel subsets of the
    configuration-0 image at passes 20..39 (the GPU renders 0..19: the samples
    are independent of the GPU's and also serve the image comparison)."""
    kind, eng = _cpu_engine()
    h = _cpu_scene_load(kind, eng, sc, "config0")
    r = cpu_render_rate(eng, h, W, H, SPP, seconds, 5, k0=SPP, seed=11, keep=True)
    eng.scene_free(h)
    threads, sample = _cpu_desc(kind, eng, r, "configuration-0 image at passes 20..39")
    return ({"value": r["value"], "unit": UNIT, "cores": threads, "kind": kind, "sample": sample,
             "median_of_subsets": r["median"]}, r["kept"])


def image_parity_config0(gs, kept):
    """Configuration 0 in expectation: the GPU's 20-pass image (passes 0..19)
    against the reference's samples of the CPU baseline (passes 20..39) per
    pixel (3-sigma band with both sides' sample variances), and both against a
    4096-pass image accumulated in FP64 on the GPU (passes 40..4135)."""
    from mupsi_b200.api import GpuRenderer
    r = GpuRenderer()
    r.prepare_render(gs)
    _, m20 = r.start_render_progressive(SPP, moments=True)
    g_mean = m20[:, :, :3] / SPP
    g_var = np.maximum(m20[:, :, 3:] / SPP - g_mean ** 2, 0.0) * SPP / (SPP - 1)
    n_ref = 4096
    _, mref = r.start_render_progressive(2 * SPP + n_ref, spp_begin=2 * SPP, moments=True)
    ref = mref[:, :, :3] / n_ref
    ref_var = np.maximum(mref[:, :, 3:] / n_ref - ref ** 2, 0.0)
    pix = np.concatenate([p for p, _ in kept])
    cpu = np.concatenate([v for _, v in kept]).astype(np.float64)
    px, py = pix % W, pix // W
    c_mean, c_var = cpu.mean(axis=1), cpu.var(axis=1, ddof=1)
    gm, gv = g_mean[py, px], g_var[py, px]
    sig = np.sqrt(gv / SPP + c_var / SPP)
    diff = gm - c_mean
    inside = np.all((np.abs(diff) <= 3 * sig) | ((sig == 0) & (diff == 0)), axis=1)
    ref_s = ref[py, px]
    rmse = float(np.sqrt(np.mean((g_mean - ref) ** 2)))
    pred = float(np.sqrt(np.mean(ref_var) * (1.0 / SPP + 1.0 / n_ref)))
    return {"workload": "configuration 0 (256x256); GPU passes 0..19, the reference's passes 20..39 on the CPU "
                        "baseline's pixels, a 4096-pass GPU image (passes 40..4135) accumulated in FP64",
            "band_pixels": int(len(pix)), "band_inside_3sigma": float(inside.mean()),
            "mean_diff_over_se": float(np.max(np.abs(diff.mean(axis=0)) /
                                              (np.sqrt(np.sum(sig ** 2, axis=0)) / len(pix) + 1e-12))),
            "rmse_gpu_20spp_vs_4096": rmse, "rmse_predicted_mc": pred,
            "rmse_gpu_20spp_vs_4096_on_subset": float(np.sqrt(np.mean((gm - ref_s) ** 2))),
            "rmse_reference_20spp_vs_4096_on_subset": float(np.sqrt(np.mean((c_mean - ref_s) ** 2))),
            "image_mean_gpu_4096": float(ref.mean())}


EXTRAS = ("config1", "config2", "config4", "config3", "next")


def run_extras(args, only=None):
    """The other configurations on the same GPU, device-timed with CUDA events:
    1 (psi microbench), 2 (level-6 mesh mean render), 4 (batched instances) and
    3 (level-8 mesh, exact mean against the surrogate), and the scene features
    beyond the configurations (image skydrome, textured mesh, SDF and external
    GP media, the progressive display). `only` runs one of them."""
    out = {}
    l2 = l2_bandwidth()
    out["l2_gbs_measured"] = l2
    legs = {"config1": ("config1_psi", run_psi_sweep), "config2": ("config2_mesh", lambda: run_mesh(l2=l2)),
            "config4": ("config4_batch", run_batch), "config3": ("config3_surrogate", lambda: run_surrogate(l2=l2)),
            "next": ("scene_features", run_scene_features)}
    for name in EXTRAS:
        if only is None or only == name:
            key, fn = legs[name]
            out[key] = fn()
    return out


def run_psi_sweep():
    """Configuration 1: psi + grad psi + Renewal+ conditioning at 2^24 points per
    sweep point (length scale x aniso x points per cell, 18 points)."""
    import torch
    from mupsi_b200.api import SparseGPNoiseGenerator, SparseSEKernel

    n = 1 << 24
    g = torch.Generator(device="cuda").manual_seed(0)
    p = (torch.rand((n, 3), device="cuda", generator=g) * 300 - 150).contiguous()
    seed = torch.randint(0, 2**31 - 1, (n,), device="cuda", generator=g, dtype=torch.int32)
    d = torch.randn((n, 3), device="cuda", generator=g)
    d = d / d.norm(dim=1, keepdim=True)
    cond = torch.zeros((n, 8), device="cuda")
    res = torch.empty((n, 4), device="cuda")
    sweep = {}
    imps = 0
    total_ms = 0.0
    for L in (0.5, 1.0, 4.0):
        for az in (1.0, 4.0):
            for ppc in (1, 3, 8):
                cond[:, :3] = p + d * torch.rand((n, 1), device="cuda", generator=g) * 3 * L
                cond[:, 3] = torch.randn(n, device="cuda", generator=g)
                gg = torch.randn((n, 3), device="cuda", generator=g)
                cond[:, 4:7] = gg / gg.norm(dim=1, keepdim=True) * torch.randn((n, 1), device="cuda", generator=g)
                cond[:, 7] = 1
                gen = SparseGPNoiseGenerator(SparseSEKernel(1.0, L, (1, 1, az)), ppc)
                for _ in range(2):
                    gen.raw_noise(p, seed, cond=cond, out=res)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                gen.raw_noise(p, seed, cond=cond, out=res)
                e1.record()
                e1.synchronize()
                ms = e0.elapsed_time(e1)
                total_ms += ms
                imps += n * 27 * ppc
                sweep[f"L{L}_aniso{az:g}_ppc{ppc}"] = {"ms": round(ms, 3), "Gqueries_s": round(n / ms / 1e6, 3)}
    peak, basis = issue_bound(OPS_PER_IMPULSE_GRAD)
    achieved = imps / (total_ms / 1e3)
    return {"queries_per_point": n, "points": 18, "total_ms": round(total_ms, 2),
            "Gimpulse_evals_s": round(imps / total_ms / 1e6, 1), "sweep": sweep,
            "roofline": {"bound": "issue", "kernel": "k_psi", "achieved": achieved / 1e9, "peak": peak / 1e9,
                         "unit": "Gimpulse-evals/s", "frac": achieved / peak, "peak_basis": basis + " (value, "
                         "gradient; the Renewal+ terms, per query, are not counted)"},
            "cpu_baseline": cpu_baseline_psi(), "gpu_Gimpulse_evals_s": achieved / 1e9}


def cpu_baseline_psi(seconds=8.0):
    """Configuration 1 on the CPU: GPMedium::evalWithGradient of the reference
    (RawNoise + Renewal+ terms over a sphere mean, OpenMP over the queries) on
    a uniform sample of each sweep point's query distribution."""
    from oracle import bind
    kind, eng = _cpu_engine()
    rng = np.random.default_rng(5)
    per = seconds / 18.0
    imps = 0
    total = 0.0
    nq = 0
    for L in (0.5, 1.0, 4.0):
        for az in (1.0, 4.0):
            for ppc in (1, 3, 8):
                k = bind.kernel_struct(1.0, L, (1, 1, az), ppc)
                n = 4096 if kind != "reference" else 0
                if kind == "reference":  # size the sample from a probe of 4096 queries
                    h = eng.medium_create(0, k, center=(0.0, 0.0, 0.0), radius=70.0)
                    pp = rng.uniform(-150, 150, (4096, 3)).astype(np.float32)
                    t = time.perf_counter()
                    eng.medium_eval(h, pp, np.arange(4096, dtype=np.uint32))
                    n = int(max(4096, 4096 * per / max(1e-6, time.perf_counter() - t)))
                    eng.medium_free(h)
                p = rng.uniform(-150, 150, (n, 3)).astype(np.float32)
                sd = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
                d = rng.normal(size=(n, 3))
                d /= np.linalg.norm(d, axis=1, keepdims=True)
                c = np.zeros((n, 8), np.float32)
                c[:, :3] = p + d * rng.uniform(0, 3 * L, (n, 1))
                c[:, 3] = rng.normal(size=n)
                g = rng.normal(size=(n, 3))
                c[:, 4:7] = g / np.linalg.norm(g, axis=1, keepdims=True) * rng.normal(size=(n, 1))
                c[:, 7] = 1
                if kind == "reference":
                    h = eng.medium_create(0, k, center=(0.0, 0.0, 0.0), radius=70.0)
                    t = time.perf_counter()
                    eng.medium_eval(h, p, sd, c)
                    total += time.perf_counter() - t
                    eng.medium_free(h)
                else:
                    t = time.perf_counter()
                    eng.psi(k, p, sd, cond=c)
                    total += time.perf_counter() - t
                imps += n * 27 * ppc
                nq += n
    model, cores = _cpu_info()
    threads = eng.num_threads() if kind == "reference" else cores
    return {"value": imps / total / 1e9, "unit": "Gimpulse-evals/s", "queries_per_s": nq / total, "cores": threads,
            "kind": kind, "sample": f"{nq} queries over the 18 sweep points (the same distributions, "
                                    f"{total:.1f} s), {threads} OpenMP threads on {model}"}


def _reference_scene(engine, sc, td, name):
    """Write what the reference's Controller::load reads for scene `sc` (OBJ
    files with texcoords, raw images, GridMeanFunction grids, scene.json) and
    load it into the reference timing build."""
    from mupsi_b200 import scene as S
    objs = []
    for i, m in enumerate(sc.meshes):
        op = os.path.join(td, f"{name}_{i}.obj")
        S.save_obj(op, m.vertices, m.faces, m.texcoords, m.face_texcoords)
        objs.append(op)
    sky_path = None
    if sc.sky_texture is not None:
        sky_path = os.path.join(td, f"{name}_sky.hdr")
        S.save_image_raw(sky_path, sc.sky_texture)
    tex = {}
    for i, pr in enumerate(sc.primitives):
        if pr.get("texture") is not None:
            tex[i] = os.path.join(td, f"{name}_tex{i}.hdr")
            S.save_image_raw(tex[i], pr["texture"])
    grids = None
    m0 = sc.media[0] if sc.media else {}
    if m0.get("kind") == "external_gp":
        m0["mean_grid"].tofile(os.path.join(td, f"{name}_mean.bin"))
        vp = None
        if m0["var_grid"] is not None:
            vp = f"{name}_var.bin"
            m0["var_grid"].tofile(os.path.join(td, vp))
        grids = (f"{name}_mean.bin", vp)
    j, extra = sc.to_json(obj_paths=objs, sky_path=sky_path, texture_paths=tex, grid_paths=grids)
    jp = os.path.join(td, f"{name}.json")
    with open(jp, "w") as fh:
        json.dump(j, fh)
    return engine.scene_load(jp, sky=None if sky_path else 1.0, extra_meshes=extra)


def run_scene_features(cpu_seconds=2.0):
    """The scene features beyond configurations 0-4 at 256x256x20 (the
    configuration-0 camera and bounce limit): GPU device time of a full render
    (median of 3 after a warm-up) and the reference's timing build on a strided
    pixel subset of the same scene; and the progressive display publishing a
    frame after every pass of the configuration-0 scene."""
    import torch
    from mupsi_b200 import scene as S
    from mupsi_b200.api import GpuDisplay, GpuRenderer, GpuScene

    rng = np.random.default_rng(31)
    sky = rng.uniform(0.2, 3.0, (128, 256, 3)).astype(np.float32)
    tex = rng.uniform(0.05, 0.95, (64, 64, 3)).astype(np.float32)
    scenes = {}
    s0 = S.config0_scene(W, H, SPP)
    s0.sky_texture = sky
    scenes["sky_texture"] = s0
    scenes["albedo_texture"] = S.textured_floor_scene(tex, True, W, H, SPP)
    for kind in ("sdf_sphere", "sdf_mesh", "external_gp"):
        scenes[kind] = S.field_scene(kind, W, H, SPP)
    kind, eng = _cpu_engine()
    td = tempfile.mkdtemp()
    out = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for name, sc in scenes.items():
        gs = GpuScene(sc)
        r = GpuRenderer()
        r.prepare_render(gs)
        fb = torch.empty((H, W, 3), device="cuda")
        r.start_render_progressive(SPP, out=fb)
        ts = []
        for _ in range(3):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            r.start_render_progressive(SPP, out=fb)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        gs.close()
        ms = float(np.median(ts))
        entry = {"gpu_ms": round(ms, 3), "gpu_samples_per_s": SAMPLES_PER_STEP / (ms / 1000.0)}
        if kind == "reference":
            with _StdoutToStderr():
                h = _reference_scene(eng, sc, td, name)
            rr = cpu_render_rate(eng, h, W, H, SPP, cpu_seconds, 2, seed=21)
            eng.scene_free(h)
            _, smp = _cpu_desc(kind, eng, rr, f"the {name} scene at all {SPP} passes")
            entry.update({"cpu_reference_samples_per_s": rr["value"], "cpu_sample": smp,
                          "gpu_over_cpu": entry["gpu_samples_per_s"] / rr["value"]})
        out[name] = entry
    # progressive display: a frame (pinned front/back swap) after every pass
    d = GpuDisplay(S.config0_scene(W, H, 64))
    d.start_progressive(2, 1)
    while d.running():
        time.sleep(0.001)
    d.stop()
    frames = 0
    t0 = time.perf_counter()
    d.start_progressive(64, 1)
    while d.running() or d.is_spp_pass_done():
        if d.is_spp_pass_done():
            d.ack_spp_pass()
            frames += 1
        time.sleep(0.0002)
    d.stop()
    wall = time.perf_counter() - t0
    out["progressive_display"] = {"workload": "configuration 0, 256x256, 64 passes, a frame after every pass",
                                  "wall_s": round(wall, 4), "passes_per_s": 64 / wall,
                                  "frames_seen_by_poller": frames, "current_spp": d.current_spp()}
    d.close()
    return out


def _timed_render(gs, w, h, spp, spp_begin=0):
    """Device time (ms) of one render of passes [spp_begin, spp) after a warm-up."""
    import torch
    from mupsi_b200.api import GpuRenderer
    r = GpuRenderer()
    r.prepare_render(gs)
    fb = torch.empty((h, w, 3), device="cuda")
    r.start_render_progressive(1, out=fb)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    r.start_render_progressive(spp, spp_begin=spp_begin, out=fb)
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1), r, fb


def _profiled(gs, r, fb, spp, bvh_spp, samples_per_pass, l2):
    """Profile stats of a render of `spp` passes (timing, work) and BVH bytes per
    sample from a counted render of `bvh_spp` passes; the march roofline."""
    gs.profile(True)
    gs.stats(reset=True)
    r.start_render_progressive(spp, out=fb)
    st = gs.stats(reset=True)
    gs.profile(False)
    bps, _ = bvh_bytes_per_sample(gs, lambda: r.start_render_progressive(bvh_spp, out=fb), bvh_spp * samples_per_pass)
    peaks, _ = _peaks()
    return march_roofline(st, spp * samples_per_pass, bvh=bps, l2_gbs=l2, hbm_gbs=float(peaks.get("hbm_gbs", 6650.0)))


def cpu_baseline_render(sc, name, w, h, spp, seconds, subsets=3, seed=3, passes=4):
    """The reference's timing build on disjoint random pixel subsets of the
    scene's image at `passes` of its passes (a sample's cost does not depend on
    its pass index; more pixels at fewer passes sample the image better in the
    few hundred samples a mesh scene allows)."""
    kind, eng = _cpu_engine()
    hd = _cpu_scene_load(kind, eng, sc, name)
    r = cpu_render_rate(eng, hd, w, h, passes, seconds, subsets, seed=seed)
    eng.scene_free(hd)
    threads, sample = _cpu_desc(kind, eng, r, f"{name} image at passes 0..{passes - 1} of {spp}")
    return {"value": r["value"], "unit": UNIT, "cores": threads, "kind": kind, "sample": sample,
            "median_of_subsets": r["median"]}


def run_mesh(l2=None):
    """Configuration 2: displaced icosphere level 6 (81,920 triangles) mesh mean, 512x512x64."""
    from mupsi_b200 import scene as S
    from mupsi_b200.api import GpuScene

    sc = S.config_mesh_scene(level=6, width=512, height=512, spp=64)
    gs = GpuScene(sc)
    ms, r, fb = _timed_render(gs, 512, 512, 64)
    n = 512 * 512 * 64
    roof = _profiled(gs, r, fb, 16, 4, 512 * 512, l2 if l2 else l2_bandwidth())
    gs.close()
    cpu = cpu_baseline_render(sc, "config2", 512, 512, 64, 12.0, passes=1)
    return {"workload": "displaced icosphere level 6 (81,920 triangles) mesh mean, 512x512x64, "
                        "length_scale 2, floor quad", "ms": round(ms, 1), "samples_per_s": n / (ms / 1000.0),
            "roofline": roof, "cpu_baseline": cpu, "gpu_over_cpu": n / (ms / 1000.0) / cpu["value"]}


def run_surrogate(spp=64, train_steps=6000, l2=None):
    """Configuration 3: the displaced icosphere at level 8 (1,310,720 triangles) as
    the mesh mean, 1024x1024x64, renewal_plus. The surrogate MLP is trained on
    the GPU on 2^22 points (half uniform in the medium's bounding box, half
    surface samples moved by N(0, 2^2) along the normal) labelled with the GPU's
    exact BVH mean, checked on 2^18 held-out points, then attached (band 3,
    scale 1.5, margin from the held-out bound violations x 2). Both forms render
    all 64 passes, device-timed. The plain every-step exact form and the lazy
    exact form are also timed on the same seeded random pixel subset of the
    same 1024x1024 image at all 64 passes (the plain form is ~100x slower)."""
    import torch
    from mupsi_b200 import scene as S
    from mupsi_b200 import surrogate as SG
    from mupsi_b200.api import GpuScene

    res = 1024
    center = np.array([0.0, 0.0, -300.0], np.float32)
    sc = S.config_mesh_scene(level=8, width=res, height=res, spp=64)
    gs = GpuScene(sc)
    mesh = sc.meshes[0]
    lo, hi = center - 100.0, center + 100.0
    t0 = time.perf_counter()
    P = SG.training_points(mesh.vertices, mesh.faces, 1 << 22, lo, hi, seed=0)
    Pd = torch.tensor(P, device="cuda")
    Td = gs.mean(0, Pd)[:, 0].contiguous()
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    Q = SG.training_points(mesh.vertices, mesh.faces, 1 << 18, lo, hi, seed=1)
    TQ = gs.mean(0, Q)[:, 0].copy()
    sm = SG.SurrogateMean(center, 32.0, seed=0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    losses = sm.train(Pd, Td, steps=train_steps, batch=16384, lr=3e-3, lr_final=1e-5, seed=0)
    e1.record()
    e1.synchronize()
    train_ms = e0.elapsed_time(e1)
    pred = sm.infer(Q)
    err = np.abs(pred - TQ)
    far = np.abs(pred) > 3.0
    margin = SG.bound_margin(pred, TQ, band=3.0, scale=1.5, safety=2.0)
    n = res * res * spp
    l2 = l2 if l2 else l2_bandwidth()

    ms_e, r_e, fb_e = _timed_render(gs, res, res, spp)
    img_e = fb_e.cpu().numpy()
    roof_e = _profiled(gs, r_e, fb_e, 4, 1, res * res, l2)
    gs2 = GpuScene(sc)
    SG.attach(gs2, 0, sm, band=3.0, scale=1.5, margin=margin, max_requests=8)
    ms_s, r_s, fb_s = _timed_render(gs2, res, res, spp)
    img_s = fb_s.cpu().numpy()
    roof_s = _profiled(gs2, r_s, fb_s, 4, 1, res * res, l2)
    gs2.profile(True)
    gs2.stats(reset=True)
    r_s.start_render_progressive(4, out=fb_s)
    st_s = gs2.stats(reset=True)
    gs2.profile(False)

    # the plain every-step form and the lazy exact form on one pixel subset of the same image
    pix = _pixel_subsets(res, res, 1024, 1, 9)[0]
    xs, ys, ks = _samples(pix, res, spp)
    gp = GpuScene(sc)
    gp.set_mean_eval(0, every_step=True)
    gp.trace(xs[:256], ys[:256], ks[:256])  # warm-up
    sub = {}
    for name, g in (("plain_every_step", gp), ("lazy_exact", gs)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        g.trace(xs, ys, ks)
        sub[name] = len(xs) / (time.perf_counter() - t)
    gp.close()
    cpu = cpu_baseline_render(sc, "config3", res, res, spp, 12.0, passes=1)
    rmse = float(np.sqrt(np.mean((img_s - img_e) ** 2)))
    out = {"workload": f"displaced icosphere level 8 (1,310,720 triangles) mesh mean, 1024x1024x{spp}, "
                       "renewal_plus, length_scale 2, floor quad",
           "training": {"points": 1 << 22, "steps": train_steps, "batch": 16384, "train_ms": round(train_ms, 1),
                        "data_s": round(t_data, 2), "final_loss": float(losses[-50:].mean())},
           "held_out": {"points": 1 << 18, "mean_abs_err": float(err.mean()), "p99_abs_err": float(np.quantile(err, .99)),
                        "max_abs_err": float(err.max()), "max_abs_err_outside_band": float(err[far].max()),
                        "bound": f"|mu| >= |m|/1.5 - {margin:.3f} outside |m| > 3"},
           "exact": {"ms": round(ms_e, 1), "samples_per_s": n / (ms_e / 1e3), "roofline": roof_e},
           "surrogate": {"ms": round(ms_s, 1), "samples_per_s": n / (ms_s / 1e3), "roofline": roof_s,
                         "predictions_per_sample": st_s["surr_requests"] / (4 * res * res),
                         "accepted_per_sample": st_s["surr_accepted"] / (4 * res * res)},
           "pixel_subset": {"workload": f"{len(pix)} seeded random pixels of the 1024x1024 image x {spp} passes "
                                        f"({len(xs)} samples, through mupsi_gpu_trace_samples, wall clock)",
                            "plain_every_step_samples_per_s": sub["plain_every_step"],
                            "lazy_exact_samples_per_s": sub["lazy_exact"],
                            "lazy_over_plain": sub["lazy_exact"] / sub["plain_every_step"]},
           "speedup": ms_e / ms_s,
           "speedup_vs_plain": (n / (ms_s / 1e3)) / sub["plain_every_step"],
           "image_rmse_vs_exact": rmse, "image_rmse_rel": rmse / max(1e-12, float(np.mean(img_e))),
           "identical_pixels": float(np.all(img_s.view(np.uint32) == img_e.view(np.uint32), axis=2).mean()),
           "cpu_baseline": cpu, "gpu_surrogate_over_cpu": (n / (ms_s / 1e3)) / cpu["value"]}
    gs2.close()
    sm.close()
    gs.close()
    return out


def run_batch():
    """Configuration 4: 64 seeded uneven sphere-mean instances (resolution 64^2..512^2,
    4-64 spp, max_bounce 2-10, length_scale U(0.25, 4), 1/3/8 points per cell, half
    single_realization) rendered as one batch: shared wave queues, one captured graph
    per bounce count, launch shapes from mupsi_b200/tuning.json. Device time from
    the batch's CUDA events (first wave start to each instance's last wave)."""
    import torch
    from mupsi_b200 import scene as S
    from mupsi_b200.api import GpuBatch, get_tuning

    scenes = S.batch_scenes(64)
    spp = [s.spp for s in scenes]
    paths = sum(s.width * s.height * s.spp for s in scenes)
    b = GpuBatch(scenes)
    b.render([max(1, k // 8) for k in spp])  # warm-up: graphs captured, buffers sized
    res = {}
    for graphs in (True, False):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, done = b.render(spp, use_graphs=graphs)
        wall = time.perf_counter() - t0
        ms = float(np.max(done))
        info = b.info()
        res["graphs" if graphs else "no_graphs"] = {
            "ms": round(ms, 2), "samples_per_s": paths / (ms / 1000.0), "wall_s": round(wall, 3),
            "waves": info["waves"], "graph_launches": info["graph_launches"]}
        if graphs:
            res["done_ms"] = [round(float(x), 2) for x in done]
    done = np.array(res["done_ms"])
    b.close()
    # the march work of every instance (the same marches as in the batch), from
    # a profiled single-scene render of each, against the batch's device time
    from mupsi_b200.api import GpuRenderer, GpuScene
    imps = 0
    for sc in scenes:
        g = GpuScene(sc)
        r = GpuRenderer()
        r.prepare_render(g)
        g.profile(True)
        r.start_render_progressive(sc.spp)
        imps += g.stats(reset=True)["impulse_evals"]
        g.close()
    peak, basis = issue_bound(OPS_PER_IMPULSE)
    achieved = imps / (res["graphs"]["ms"] / 1e3)
    cpu = cpu_baseline_batch(scenes)
    return {"workload": "64 instances of batch_scenes(seed 4): res {64..512}^2, spp 4-64, max_bounce 2-10, "
                        "length U(0.25,4), ppc {1,3,8}, sphere mean r U(20,100) in 1.8r null sphere, "
                        "half single_realization", "path_samples": paths,
            "samples_per_s": res["graphs"]["samples_per_s"], "ms": res["graphs"]["ms"],
            "completion_ms": {"min": float(done.min()), "median": float(np.median(done)),
                              "max": float(done.max()), "mean": float(done.mean())},
            "roofline": {"bound": "issue", "kernel": "k_march", "achieved": achieved / 1e9, "peak": peak / 1e9,
                         "unit": "Gimpulse-evals/s", "frac": achieved / peak, "peak_basis": basis,
                         "note": "impulse evaluations counted per instance in profiled single-scene renders "
                                 "(the same marches) over the batch's device time (march + shade + raygen)"},
            "cpu_baseline": cpu, "gpu_over_cpu": res["graphs"]["samples_per_s"] / cpu["value"],
            "tuning": get_tuning(), **res}


def cpu_baseline_batch(scenes, samples_per_instance=384):
    """Configuration 4 on the CPU: each instance's rate from the reference's
    timing build on a seeded random pixel subset at all of the instance's
    passes; the instances' full renders timed as their samples over those
    rates, summed (the reference renders one scene at a time)."""
    kind, eng = _cpu_engine()
    t_sum, n_sum, n_traced, t_traced = 0.0, 0, 0, 0.0
    for i, sc in enumerate(scenes):
        hd = _cpu_scene_load(kind, eng, sc, f"batch{i}")
        npix = max(1, samples_per_instance // sc.spp)
        pix = _pixel_subsets(sc.width, sc.height, npix, 1, 100 + i)[0]
        xs, ys, ks = _samples(pix, sc.width, sc.spp)
        t = time.perf_counter()
        eng.trace(hd, xs, ys, ks)
        dt = time.perf_counter() - t
        eng.scene_free(hd)
        paths = sc.width * sc.height * sc.spp
        t_sum += paths * dt / len(xs)
        n_sum += paths
        n_traced += len(xs)
        t_traced += dt
    model, cores = _cpu_info()
    threads = eng.num_threads() if kind == "reference" else cores
    return {"value": n_sum / t_sum, "unit": UNIT, "cores": threads, "kind": kind,
            "estimated_full_batch_s": t_sum,
            "sample": f"per instance ~{samples_per_instance} samples (random pixels x all passes), {n_traced} in "
                      f"{t_traced:.1f} s; full-batch time = sum over instances of samples / rate; {threads} "
                      f"OpenMP threads on {model}"}


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
    elif args.only:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        print(json.dumps(run_extras(args, only=args.only)), flush=True)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
