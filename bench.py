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
restatement of the oracle when that library is absent) on a strided pixel
subset of the same scene at all 20 passes, with every host thread.
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
    ap.add_argument("--cpu-seconds", type=float, default=8.0, help="CPU work per reference/baseline step")
    ap.add_argument("--extras", type=int, default=1, help="also time configurations 1-4 (single GPU)")
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


def _cpu_scene(engine_kind, engine, scene):
    if engine_kind == "reference":
        td = tempfile.mkdtemp()
        j, _ = scene.to_json()
        jp = os.path.join(td, "config0.json")
        with open(jp, "w") as fh:
            json.dump(j, fh)
        return engine.scene_load(jp, sky=1.0)
    return engine.scene_create(scene.desc())


def _cpu_samples(n, offset=0):
    """n samples on a strided pixel subset, every pass of each pixel."""
    npix = max(1, n // SPP)
    stride = max(1, (W * H) // npix) | 1  # odd: the subset spreads over columns and rows
    pix = (np.arange(npix) * stride + offset) % (W * H)
    xs = np.repeat(pix % W, SPP).astype(np.int32)
    ys = np.repeat(pix // W, SPP).astype(np.int32)
    ks = np.tile(np.arange(SPP, dtype=np.int32), npix)
    return xs, ys, ks, stride


def cpu_rate(seconds, scene, steps=1, warmup=0):
    """Time the CPU implementation on bounded strided samples; returns a dict."""
    kind, eng = _cpu_engine()
    h = _cpu_scene(kind, eng, scene)
    xs, ys, ks, _ = _cpu_samples(SPP * 256)
    t = time.perf_counter()
    eng.trace(h, xs, ys, ks)
    rate0 = len(xs) / (time.perf_counter() - t)
    n = int(max(SPP * 16, rate0 * seconds))
    times = []
    for i in range(warmup + steps):
        xs, ys, ks, stride = _cpu_samples(n, offset=i)
        t = time.perf_counter()
        eng.trace(h, xs, ys, ks)
        if i >= warmup:
            times.append(time.perf_counter() - t)
    model, cores = _cpu_info()
    threads = eng.num_threads() if kind == "reference" else cores
    return {"value": len(xs) * len(times) / sum(times), "kind": kind, "cores": threads, "n": len(xs),
            "stride": stride, "seconds": sum(times), "model": model,
            "sample": f"{len(xs)} path samples per step: every {stride}th pixel (row-major) x all {SPP} passes of "
                      f"the configuration-0 scene, {threads} OpenMP threads on {model}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from mupsi_b200 import scene as S
    r = cpu_rate(args.cpu_seconds, S.config0_scene(W, H, SPP), steps=args.steps, warmup=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * r["n"] / r["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": _config({"parallelism": "openmp", "sample": r["sample"]}),
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                             "sample": r["sample"]},
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


def _profiled_traffic():
    """dram read + write bytes of the profiled k_march launch (profiles/k_march_config0.md)."""
    try:
        for line in open(os.path.join(ROOT, "profiles", "k_march_config0.md")):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":", 1)[1])
    except (OSError, ValueError):
        pass
    return None


# Source-level operations per impulse evaluation of the march's psi sum (the
# roofline unit): 4 PCG32 steps at 10 integer ops each (64-bit multiply-add as
# three 32-bit multiply-adds plus carry, xorshift, rotate), 3 mantissa-trick
# uniforms for the position (shift/or, subtract: 1 integer + 1 float each), the
# weight's sign bit put onto the Gaussian (1 three-input logic op), the impulse
# position (3 multiply + 3 add), |p - s|^2 (3 sub, 1 mul, 2 fused multiply-add),
# the exponent scale (1 mul), exp2 on the SFU (1), the signed accumulate (1 add):
# 44 integer + 18 float = 62 issue slots, 1 of them on the SFU.
OPS_PER_IMPULSE = 62


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
    peaks, peak_kind = _peaks()
    mhz = float(peaks.get("sm_max_mhz", 1965.0))
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    peak_gimp = sms * 4 * 32 * mhz * 1e6 / OPS_PER_IMPULSE / 1e9  # 4 schedulers x 32 lanes, 1 issue/clock
    achieved = st["impulse_evals"] / (st["march_ms"] / 1000.0) / 1e9 if st["march_ms"] > 0 else 0.0
    roof = {"bound": "issue", "kernel": "k_march", "achieved": achieved, "peak": peak_gimp,
            "unit": "Gimpulse-evals/s", "frac": achieved / peak_gimp, "traffic": _profiled_traffic(),
            "traffic_note": "DRAM bytes of the bounce-1 k_march launch from profiles/k_march_config0.md",
            "peak_basis": f"{sms} SMs x 128 lanes x {mhz:.0f} MHz ({peak_kind} sm_max_mhz) / {OPS_PER_IMPULSE} "
                          f"ops per impulse", "march_share": st["march_ms"] / max(1e-9, st["march_ms"] + st["shade_ms"]),
            "launches": st["march_launches"], "ms_per_launch": st["march_ms"] / max(1, st["march_launches"]),
            "impulse_evals_per_launch": st["impulse_evals"] / max(1, st["march_launches"]),
            "psi_evals_per_sample": st["psi_evals"] / (2.0 * SAMPLES_PER_STEP),
            "march_steps_per_sample": st["march_steps"] / (2.0 * SAMPLES_PER_STEP)}

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

    cpu = None
    if rank == 0 and world == 1:
        r = cpu_rate(args.cpu_seconds, sc, steps=1, warmup=0)
        cpu = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"], "sample": r["sample"]}
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
        if extras:
            line["extras"] = extras
        print(json.dumps(line), flush=True)
    gs.close()
    if world > 1:
        dist.destroy_process_group()


EXTRAS = ("config1", "config2", "config4", "config3", "next")


def run_extras(args, only=None):
    """The other configurations on the same GPU, device-timed with CUDA events:
    1 (psi microbench), 2 (level-6 mesh mean render), 4 (batched instances) and
    3 (level-8 mesh, exact mean against the surrogate), and the scene features
    beyond the configurations (image skydrome, textured mesh, SDF and external
    GP media, the progressive display). `only` runs one of them."""
    out = {}
    legs = {"config1": ("config1_psi", run_psi_sweep), "config2": ("config2_mesh", run_mesh),
            "config4": ("config4_batch", run_batch), "config3": ("config3_surrogate", run_surrogate),
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
    return {"queries_per_point": n, "points": 18, "total_ms": round(total_ms, 2),
            "Gimpulse_evals_s": round(imps / total_ms / 1e6, 1), "sweep": sweep}


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
            h = _reference_scene(eng, sc, td, name)
            xs, ys, ks, _ = _cpu_samples(SPP * 256)  # 256 pixels on the image's diagonal: a fair rate estimate
            t = time.perf_counter()
            eng.trace(h, xs, ys, ks)
            rate0 = len(xs) / (time.perf_counter() - t)
            xs, ys, ks, stride = _cpu_samples(int(max(SPP * 64, rate0 * cpu_seconds)), offset=1)
            t = time.perf_counter()
            eng.trace(h, xs, ys, ks)
            cpu = len(xs) / (time.perf_counter() - t)
            eng.scene_free(h)
            entry.update({"cpu_reference_samples_per_s": cpu, "cpu_sample": f"{len(xs)} samples, every {stride}th "
                          f"pixel x {SPP} passes, {eng.num_threads()} threads", "gpu_over_cpu": entry["gpu_samples_per_s"] / cpu})
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


def run_mesh():
    """Configuration 2: displaced icosphere level 6 (81,920 triangles) mesh mean, 512x512x64."""
    import torch
    from mupsi_b200 import scene as S
    from mupsi_b200.api import GpuRenderer, GpuScene

    sc = S.config_mesh_scene(level=6, width=512, height=512, spp=64)
    gs = GpuScene(sc)
    r = GpuRenderer()
    r.prepare_render(gs)
    fb = torch.empty((512, 512, 3), device="cuda")
    r.start_render_progressive(2, out=fb)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    r.start_render_progressive(64, out=fb)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    gs.close()
    return {"workload": "displaced icosphere level 6 (81,920 triangles) mesh mean, 512x512x64, "
                        "length_scale 2, floor quad", "ms": round(ms, 1), "samples_per_s": 512 * 512 * 64 / (ms / 1000.0)}


def run_surrogate(spp=2, train_steps=6000):
    """Configuration 3: the displaced icosphere at level 8 (1,310,720 triangles) as
    the mesh mean, 1024x1024, renewal_plus. The surrogate MLP is trained on the
    GPU on 2^22 points (half uniform in the medium's bounding box, half surface
    samples moved by N(0, 2^2) along the normal) labelled with the GPU's exact
    BVH mean, checked on 2^18 held-out points, then attached (band 3, scale 1.5,
    margin from the held-out bound violations x 2). Both forms render the same
    `spp` passes (a bounded sample of the 64-spp workload), device-timed, best of
    two renders."""
    import torch
    from mupsi_b200 import scene as S
    from mupsi_b200 import surrogate as SG
    from mupsi_b200.api import GpuRenderer, GpuScene

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

    def render(g):
        r = GpuRenderer()
        r.prepare_render(g)
        fb = torch.empty((res, res, 3), device="cuda")
        r.start_render_progressive(1, out=fb)  # warm-up
        g.profile(True)
        g.stats(reset=True)
        times = []
        for _ in range(2):  # best of two renders of the same passes
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            r.start_render_progressive(spp, out=fb)
            b.record()
            b.synchronize()
            times.append(a.elapsed_time(b))
        st = g.stats(reset=True)
        g.profile(False)
        st = {k: (v / 2 if isinstance(v, (int, float)) else v) for k, v in st.items()}  # per render
        return fb.cpu().numpy(), min(times), st

    img_e, ms_e, st_e = render(gs)
    # the plain exact form (BVH parity cast + closest point at every visited
    # step) on a 256x256 view of the same scene: same rays per pixel sample,
    # 16x fewer samples to keep the run short
    scp = S.config_mesh_scene(level=8, width=256, height=256, spp=2)
    gp = GpuScene(scp)
    gp.set_mean_eval(0, every_step=True)
    rp = GpuRenderer()
    rp.prepare_render(gp)
    fbp = torch.empty((256, 256, 3), device="cuda")
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    rp.start_render_progressive(2, out=fbp)
    b.record()
    b.synchronize()
    plain_ms = a.elapsed_time(b)
    plain_rate = 256 * 256 * 2 / (plain_ms / 1e3)
    gp.close()
    gs2 = GpuScene(sc)
    SG.attach(gs2, 0, sm, band=3.0, scale=1.5, margin=margin, max_requests=8)
    img_s, ms_s, st_s = render(gs2)
    n = res * res * spp
    rmse = float(np.sqrt(np.mean((img_s - img_e) ** 2)))
    out = {"workload": f"displaced icosphere level 8 (1,310,720 triangles) mesh mean, 1024x1024, {spp} of 64 spp, "
                       "renewal_plus, length_scale 2, floor quad",
           "training": {"points": 1 << 22, "steps": train_steps, "batch": 16384, "train_ms": round(train_ms, 1),
                        "data_s": round(t_data, 2), "final_loss": float(losses[-50:].mean())},
           "held_out": {"points": 1 << 18, "mean_abs_err": float(err.mean()), "p99_abs_err": float(np.quantile(err, .99)),
                        "max_abs_err": float(err.max()), "max_abs_err_outside_band": float(err[far].max()),
                        "bound": f"|mu| >= |m|/1.5 - {margin:.3f} outside |m| > 3"},
           "exact": {"ms": round(ms_e, 1), "samples_per_s": n / (ms_e / 1e3),
                     "exact_mean_evals_per_sample": st_e["mean_evals"] / n},
           "surrogate": {"ms": round(ms_s, 1), "samples_per_s": n / (ms_s / 1e3),
                         "exact_mean_evals_per_sample": st_s["mean_evals"] / n,
                         "predictions_per_sample": st_s["surr_requests"] / n,
                         "accepted_per_sample": st_s["surr_accepted"] / n},
           "plain_every_step": {"workload": "same scene and camera at 256x256, 2 spp", "ms": round(plain_ms, 1),
                                "samples_per_s": plain_rate},
           "speedup": ms_e / ms_s,
           "speedup_vs_plain": (n / (ms_s / 1e3)) / plain_rate,
           "image_rmse_vs_exact": rmse, "image_rmse_rel": rmse / max(1e-12, float(np.mean(img_e))),
           "identical_pixels": float(np.all(img_s.view(np.uint32) == img_e.view(np.uint32), axis=2).mean())}
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
    return {"workload": "64 instances of batch_scenes(seed 4): res {64..512}^2, spp 4-64, max_bounce 2-10, "
                        "length U(0.25,4), ppc {1,3,8}, sphere mean r U(20,100) in 1.8r null sphere, "
                        "half single_realization", "path_samples": paths,
            "samples_per_s": res["graphs"]["samples_per_s"], "ms": res["graphs"]["ms"],
            "completion_ms": {"min": float(done.min()), "median": float(np.median(done)),
                              "max": float(done.max()), "mean": float(done.mean())},
            "tuning": get_tuning(), **res}


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
