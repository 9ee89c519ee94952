"""Autotuner for the wave kernels' launch shapes.

    python -m mupsi_b200.autotune [--out mupsi_b200/tuning.json] [--spp-div 4] [--passes 2]

Tunes the persistent march's block size, the smallest lane group per ray, the
shading block size, the paths per wave (the queue tile) and the queue size
per block below which sphere-mean rays are marched one per block by coordinate
descent on two workloads: a batched render of the seeded uneven instances of
scene.batch_scenes (pass counts divided by --spp-div to keep a trial short)
and the 256x256x20 configuration-0 render. Both are timed on the device with
CUDA events (the batch by its per-instance completion events, its time being
the last instance's completion), each the median of --repeats renders after
one warm-up; a candidate's score is the mean of its two times relative to the
starting shapes' times. Launch shapes do not change any result
(psi sums are added in one fixed order for every lane-group size), so every
candidate renders the same images. Writes the chosen shapes and every trial to
a JSON file that mupsi_b200.api applies when the first scene is created.
"""
import argparse
import json
import os
import time

import numpy as np

CANDIDATES = {
    "march_block": [64, 96, 128],
    "min_group": [4, 8, 16, 32],
    "shade_block": [64, 128],
    "wave_paths": [1 << 21, 1 << 22, 1 << 23, 1 << 24],
    "block_rays": [0, 4, 8, 12, 16, 24],
    "lane_rays": [0, 1, 2, 4],
    # mesh means only, which the tuning workload does not hold: the measured
    # choice (a level-6 mesh is faster one ray per lane, a level-8 mesh with
    # lane groups)
    "lane_max_tris": [1 << 18],
    # the same (measured on the level-6 mesh render at 512^2 x 8 with the
    # one-ray-per-lane mesh march at 16 blocks per SM: 8 / 16 / 24 / 32 ->
    # 248 / 232 / 227 / 227 ms)
    "mu_batch": [24],
}
DEFAULT = {"march_block": 128, "min_group": 4, "shade_block": 128, "wave_paths": 1 << 23, "block_rays": 8,
           "lane_rays": 1, "lane_max_tris": 1 << 18, "mu_batch": 24}


def coordinate_descent(measure, candidates=CANDIDATES, start=DEFAULT, passes=2):
    """Minimise measure(config) one parameter at a time, `passes` sweeps over
    the parameters. Returns (best config, best time, trials)."""
    best = dict(start)
    trials = []
    cache = {}

    def run(cfg):
        key = tuple(sorted(cfg.items()))
        if key not in cache:
            cache[key] = measure(cfg)
            trials.append({"config": dict(cfg), "value": cache[key]})
        return cache[key]

    best_t = run(best)
    for _ in range(passes):
        changed = False
        for name, values in candidates.items():
            for v in values:
                cfg = dict(best, **{name: v})
                t = run(cfg)
                if t < best_t:
                    best, best_t, changed = cfg, t, True
        if not changed:
            break
    return best, best_t, trials


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json"))
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--spp-div", type=int, default=4)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--passes", type=int, default=2)
    args = ap.parse_args(argv)

    import torch

    from . import scene as S
    from .api import GpuBatch, GpuRenderer, set_tuning

    scenes = S.batch_scenes(args.instances)
    spp = [max(1, s.spp // args.spp_div) for s in scenes]
    batch = GpuBatch(scenes)
    paths = sum(s.width * s.height * k for s, k in zip(scenes, spp))
    rend = GpuRenderer()
    rend.prepare_render(S.config0_scene(256, 256, 20))
    fb = torch.empty((256, 256, 3), dtype=torch.float32, device="cuda")
    base = {}

    def time_c0():
        rend.start_render_progressive(20, out=fb)
        ts = []
        for _ in range(args.repeats * 3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            rend.start_render_progressive(20, out=fb)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    def measure(cfg):
        set_tuning(**cfg)
        batch.render(spp)  # warm-up (and graph capture)
        ts = []
        for _ in range(args.repeats):
            _, done = batch.render(spp)
            ts.append(float(np.max(done)))
        t_batch = float(np.median(ts))
        t_c0 = time_c0()
        if not base:
            base.update(batch=t_batch, c0=t_c0)
        score = 0.5 * (t_batch / base["batch"] + t_c0 / base["c0"])
        print(json.dumps({"config": cfg, "batch_ms": round(t_batch, 3), "config0_ms": round(t_c0, 3),
                          "score": round(score, 4)}), flush=True)
        return score

    t0 = time.time()
    best, best_score, trials = coordinate_descent(measure, passes=args.passes)
    set_tuning(**best)
    out = {
        "tuning": best,
        "score": best_score,
        "baseline_ms": base,
        "device": torch.cuda.get_device_name(0),
        "workload": f"batch_scenes({args.instances}) with spp // {args.spp_div} ({paths} path samples) and the "
                    f"256x256x20 configuration-0 render",
        "tuning_seconds": round(time.time() - t0, 1),
        "trials": trials,
    }
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps({"chosen": best, "score": best_score}))
    batch.close()


if __name__ == "__main__":
    main()
