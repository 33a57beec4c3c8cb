#!/usr/bin/env python
"""Forward+backward throughput of the B200 differentiable path tracer.

Default workload: the glossy heightfield configuration -- a 256 x 256-vertex
grid (130,050 triangles in 64 patches of their own Blinn-Phong material,
heights from 6 seeded sinusoid octaves) under two area lights (4 triangles),
640 x 480, 64 spp, max_bounces 3.  Its image is rendered as 16 batches of
4 spp, one batch per step: a step renders the batch forward and runs the full
backward (path adjoints, secondary edges over the edge trees, primary edges)
against an all-ones image adjoint, with its own seed.  Per-sample work does not
depend on how a pixel's samples are batched (each pixel sample draws its own
streams and its primary-edge samples scale with it); the line reports a
measured check of that (`spp_linearity`).  Metric: pixel samples per second
(fwd+bwd); `forward` gives forward-only samples per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload heightfield|soft_shadow|single_triangle|heightfield_ggx]

N > 1 runs under torchrun; every rank renders its own replica of the workload
(samples are independent; no collective on the data path), and `value` is the
sum over ranks, timed as the max over ranks.  `--impl reference` times the
reference's own CPU renderer (oracle/_ref, compiled from the reference sources
with their flags) on this machine's cores on a bounded sample of the workload.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd samples/s"
UNIT = "samples/s"
# spp: samples per pixel of the configuration's image; step_spp: the batch one
# step renders (spp / step_spp steps make an image).  ref_res, ref_spp: the
# reference CPU arm's bounded sample per step -- the same view at a lower
# resolution (per-sample work does not depend on the resolution; its time is
# linear in samples, and the arm reports a check of that).
WORKLOADS = {
    "heightfield": dict(builder="heightfield", resolution=(640, 480), spp=64, step_spp=4, max_bounces=3,
                        scene_seed=0, ref_res=(160, 120), ref_spp=1,
                        name="glossy heightfield (130,054 triangles, Blinn-Phong)"),
    "soft_shadow": dict(builder="soft_shadow", resolution=(512, 512), spp=16, step_spp=16, max_bounces=1,
                        scene_seed=0, ref_res=(512, 512), ref_spp=16, name="soft shadow (8 triangles)"),
    "single_triangle": dict(builder="single_triangle", resolution=(256, 256), spp=4, step_spp=4, max_bounces=1,
                            scene_seed=0, ref_res=(256, 256), ref_spp=4, name="single triangle (3 triangles)"),
    # the heightfield with GGX lobes; the reference has no GGX material, so
    # its arm reports this workload unavailable
    "heightfield_ggx": dict(builder="heightfield", resolution=(640, 480), spp=64, step_spp=4, max_bounces=3,
                            scene_seed=0, ref_res=None, ref_spp=None, options={"microfacet": "ggx"},
                            name="glossy heightfield (130,054 triangles, GGX)",
                            no_reference="the reference's materials are Blinn-Phong only (no GGX lobe)"),
}
DEFAULT_WORKLOAD = "heightfield"
WORKLOAD = WORKLOADS[DEFAULT_WORKLOAD]
# reference CPU arm: page-in / warm-up steps on a small slice of the same scene
REF_RES = (32, 32)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-proposal", action="store_true", help="skip the learned-vs-plain edge sampling measurement")
    p.add_argument("--proposal-seeds", type=int, default=32, help="seeds per arm of the learned-vs-plain measurement")
    p.add_argument("--proposal-train", type=int, default=60, help="training calls before the learned arm")
    p.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    p.add_argument("--res", type=int, nargs=2, default=None, metavar=("W", "H"),
                   help="render this size instead of the workload's (smaller cases for ncu captures)")
    p.add_argument("--step-spp", type=int, default=None, help="samples per pixel of one step instead of the workload's")
    p.add_argument("--no-inverse", action="store_true", help="skip the inverse-rendering loop measurement")
    p.add_argument("--inverse-steps", type=int, default=200, help="Adam steps per arm of the inverse-rendering loop")
    return p.parse_args()


def dist_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def build_workload(res=None, spp=None):
    """The workload's scene; spp defaults to one step's batch."""
    from delta_ray_b200 import workloads
    w = WORKLOAD
    return workloads.BUILDERS[w["builder"]](seed=w["scene_seed"], resolution=res or w["resolution"],
                                            spp=spp or w["step_spp"], max_bounces=w["max_bounces"],
                                            **w.get("options", {}))


def workload_label():
    w = WORKLOAD
    batches = w["spp"] // w["step_spp"]
    per = f" as {batches} steps of {w['step_spp']} spp" if batches > 1 else ""
    return (f"{w['name']}: {w['resolution'][0]}x{w['resolution'][1]}, {w['spp']} spp{per}, "
            f"max_bounces={w['max_bounces']}, fwd+bwd")


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
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
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
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
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic work model (bytes a launch must move at minimum)
# ---------------------------------------------------------------------------
def ray_bytes(num_tris):
    """Per ray: origin+direction 24 B, hit record 16 B, 3 vertices 36 B and one
    64-B node pair per BVH level (ceil(log2 T) levels)."""
    return 24 + 16 + 36 + 64 * max(1, math.ceil(math.log2(max(2, num_tris))))


# bytes per shading vertex: path state read/write (32) + material record (28)
SHADE_BYTES = 32 + 28
# a shading-point record as the edge kernels read it (24 floats)
POINT_BYTES = 96
# an edge-tree node (edge_tree.h:12-22)
NODE_BYTES = 40


def kernel_bytes(kernel, wl, work):
    """Algorithmic bytes of one launch of `kernel` (the survey's fixed model:
    rays at ray_bytes(T) each, shading vertices at SHADE_BYTES, point records,
    items (20 B), edge-tree nodes visited (40 B), queue records, gradient
    scatter), from the call's measured work counts (Scene.last_work) and the
    pixel samples n = W * H * spp.  0 for kernels outside the model."""
    W, H = wl.resolution
    spp, B = wl.spp, wl.max_bounces
    br = ray_bytes(wl.num_triangles)
    n = W * H * spp
    P, I = work["points"], work["items"]
    rays_path = 1 + 2 * B  # upper bound: camera ray, then a shadow and a BSDF ray per bounce
    # an edge sample's shading: two shadow rays to the emitters, plus the
    # multi-bounce paths of both sides when B > 1 (1 + 2 (B - 1) rays each)
    shade_rays = 2 + (2 * (1 + 2 * (B - 1)) if B > 1 else 0)
    if kernel == "k_render_forward":
        return n * (rays_path * br + B * SHADE_BYTES) + W * H * 12
    if kernel == "k_backward_paths":
        return n * (rays_path * br + B * SHADE_BYTES) + W * H * 24 + P * POINT_BYTES
    if kernel == "k_primary_shade":  # two camera rays, two shaded paths, the 16-B color difference out
        return n * (2 * rays_path * br + 2 * B * SHADE_BYTES + 24 + 16)
    if kernel == "k_primary_grad":  # the color difference in, edge vertices, vertex and camera adds
        return n * (16 + 24 + 24)
    if kernel == "k_edge_traverse":
        return P * POINT_BYTES + I * 20 + work["visits_walk"] * NODE_BYTES
    if kernel == "k_edge_expand":
        return P * POINT_BYTES + work["items_first_stage"] * 20 + work["tasks"] * 24 + work["visits_walk"] * NODE_BYTES
    if kernel == "k_edge_tasks":
        return (work["tasks"] * (24 + POINT_BYTES) + (I - work["items_first_stage"]) * 20 +
                work["visits_tasks"] * NODE_BYTES)
    # the level walk of the same subtrees: the points' contexts, the subtrees'
    # nodes, the items of their leaves
    if kernel == "k_walk_ctx":
        return P * POINT_BYTES
    if kernel == "k_edge_level":
        return work["tasks"] * 24 + work["visits_tasks"] * NODE_BYTES
    if kernel == "k_edge_leaves":
        return (I - work["items_first_stage"]) * 20
    if kernel == "k_edge_line":  # item, point record, LTC matrix, material; survivor record out
        return I * (20 + POINT_BYTES + 36 + 28) + work["survivors"] * 32
    if kernel == "k_edge_connect":  # survivor in, the two rays' connectivity, candidate record out
        return work["survivors"] * (32 + 2 * br) + work.get("candidates", 0) * 16
    if kernel == "k_edge_pairs":  # candidate in, the other side's closest hit, hit record out
        return work.get("candidates", 0) * (16 + 32 + br + 16)
    if kernel == "k_edge_line_rays":
        return I * (20 + POINT_BYTES + 36 + 28) + work["survivors"] * 2 * br + work["shaded"] * 48
    if kernel == "k_edge_shade":  # records in, shading rays and vertices, dp out, vertex gradient adds
        return work["shaded"] * (48 + POINT_BYTES + shade_rays * br + 2 * SHADE_BYTES + 12 + 2 * 12)
    if kernel == "k_dp_propagate":
        return P * (POINT_BYTES + 36 + 12 * 3)
    return 0


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_bf16_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


# the learned proposal's network: 2 * (10*64 + 64*64 + 64*64 + 64*32) FLOP per query
MLP_FLOP_PER_QUERY = 21760


def measure_proposal(dev, K=32, train_calls=60):
    """Gradient variance x time, learned vs plain edge sampling, on two scenes:
    the glossy heightfield configuration's full mesh (130,054 triangles, 64
    patches, B = 3) at 160 x 120, 1 spp, and a small heightfield (10 x 10
    grid, 162 triangles, 96 x 72, 4 spp, B = 1, 3K seeds).  Per scene: K seeds of plain
    sampling, K more as a noise calibration (plain vs plain), `train_calls`
    backward calls of online training, then K seeds with the trained proposal.
    Per parameter the variance ratio is var_learned / var_plain; its geometric
    mean over the parameters is the statistic (the sum of variances is
    dominated by rare huge samples of the reference's edge estimator: two plain
    runs can differ by 10x in it; it is reported beside, with its plain-vs-plain
    spread).  Backward times come from CUDA events."""
    import numpy as np
    import torch
    from delta_ray_b200 import _abi, proposal, workloads
    from delta_ray_b200.render_pytorch import RenderOptions, Scene

    def small_heightfield():
        return workloads.heightfield(seed=8, resolution=(96, 72), spp=4, max_bounces=1, grid=10, patch=10)

    cases = [("glossy heightfield configuration's mesh (130,054 triangles), 160x120, 1 spp, max_bounces=3",
              lambda: workloads.heightfield(seed=0, resolution=(160, 120), spp=1, max_bounces=3), K),
             ("heightfield 10x10-vertex grid (162 triangles), 96x72, 4 spp, max_bounces=1", small_heightfield, 3 * K)]
    out = {"gradient": "image sum, dp_mode sum", "mix": 0.8, "train_calls": train_calls,
           "statistic": "geometric mean over parameters of var_learned / var_plain", "higher_is_better": False,
           "scenes": []}
    peak, kind = load_bf16_peak()
    for label, make, k_seeds in cases:
        wl = make()
        W, H = wl.resolution
        cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
        sc = Scene(cam, mats, shps, lts, dev.index or 0)
        d = torch.ones((H, W, 3), device=dev)

        def run(seeds, learned):
            opts = RenderOptions(dp_mode=_abi.DR_DP_SUM, learned_proposal=learned)
            res, ms = [], 0.0
            for s_ in seeds:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                g, _ = sc.backward(W, H, wl.spp, wl.max_bounces, s_, d, opts)
                b.record()
                torch.cuda.synchronize()
                ms += a.elapsed_time(b)
                res.append(g.cpu().numpy())
            return np.stack(res), ms / len(seeds)

        def ratios(ga, gb):
            va, vb = ga.var(0, ddof=1), gb.var(0, ddof=1)
            m = (va > 0) & (vb > 0)
            return float(np.exp(np.log(vb[m] / va[m]).mean())), float(vb.sum() / va.sum()), int(m.sum())

        try:
            run([1, 2], False)
            g_plain, t_plain = run(range(100, 100 + k_seeds), False)
            g_cal, _ = run(range(100000, 100000 + k_seeds), False)
            sc.set_proposal(train=True, mix=0.8, learning_rate=3e-3, train_points=16384,
                            params=proposal.init_params(1))
            losses = []
            for k in range(train_calls):
                run([500 + k], True)
                losses.append(sc.proposal_state()[1])
            sc.set_proposal(train=False, mix=0.8)
            run([3, 4], True)
            g_learn, t_learn = run(range(200000, 200000 + k_seeds), True)
            geo, sum_r, nparams = ratios(g_plain, g_learn)
            cal_geo, cal_sum, _ = ratios(g_plain, g_cal)
            K2 = min(k_seeds, g_plain.shape[0])
            se = np.sqrt((g_plain.var(0, ddof=1) + g_learn.var(0, ddof=1)) / K2)
            mm = se > 1e-3 * se.max()
            z = (g_learn.mean(0) - g_plain.mean(0))[mm] / se[mm]
            sc.set_profiling(True)
            sc.backward(W, H, wl.spp, wl.max_bounces, 9, d,
                        RenderOptions(dp_mode=_abi.DR_DP_SUM, learned_proposal=True))
            stages = dict(sc.last_timings())
            queries = sc.last_counts()[0]
            sc.set_profiling(False)
            infer_ms = stages.get("k_mlp_infer", 0.0)
            tflops = queries * MLP_FLOP_PER_QUERY / (infer_ms / 1e3) / 1e12 if infer_ms > 0 else 0.0
            out["scenes"].append({
                "workload": label, "seeds": k_seeds,
                "train_loss_first_last": [round(float(np.mean(losses[:3])), 4), round(float(np.mean(losses[-3:])), 4)],
                "variance_ratio": round(geo, 4), "variance_sum_ratio": round(sum_r, 4), "params_compared": nparams,
                "noise_plain_vs_plain": {"variance_ratio": round(cal_geo, 4), "variance_sum_ratio": round(cal_sum, 4)},
                "mean_difference_rms_z": round(float(np.sqrt((z ** 2).mean())), 3),
                "backward_ms": {"plain": round(t_plain, 3), "learned": round(t_learn, 3)},
                "var_x_time_ratio": round(geo * t_learn / t_plain, 4),
                "mlp_infer": {"queries": int(queries), "ms": round(infer_ms, 4), "achieved_tflops": round(tflops, 3),
                              "peak_tflops": peak, "peak_kind": kind, "frac": tflops / peak,
                              "flop_per_query": MLP_FLOP_PER_QUERY}})
        finally:
            sc.close()
    return out


def load_profile(kernel):
    """DRAM bytes and L2 figures per launch of `kernel` on this workload from
    the committed ncu summary profiles/kernels_<workload>.txt ("<kernel>
    <dram bytes> <l2 hit %> <l2 throughput % of peak> <units>" lines; the
    capture may be of a smaller case of the same scene, so its DRAM bytes are
    scaled by the units processed: samples, or the items of the call), if any."""
    if WORKLOAD_KEY is None:
        return None
    path = os.path.join(ROOT, "profiles", f"kernels_{WORKLOAD_KEY}.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 5 and parts[0] == kernel and not line.startswith("#"):
                    return {"dram_bytes": int(parts[1]), "l2_hit_pct": float(parts[2]),
                            "l2_throughput_pct": float(parts[3]), "units": int(parts[4]),
                            "source": os.path.relpath(path, ROOT)}
    except (OSError, ValueError):
        return None
    return None


WORKLOAD_KEY = DEFAULT_WORKLOAD


def measure_inverse(steps):
    """The inverse-rendering loop (delta_ray_b200.inverse) at its reduced
    setting, plain and with the learned edge proposal: a 64 x 64 height grid
    (16 roughness patches) fit to 4 views of 128 x 96 rendered at 64 spp, Adam
    (lr 3e-3) at 8 spp per view per step, direct lighting (FitConfig's
    defaults); parameter RMSE over the heights and roughness, the time to
    reach RMSE 0.01, the image loss of the first and last step."""
    from delta_ray_b200.inverse import FitConfig, fit
    out = {"setting": "64x64-vertex heightfield (7,938 triangles + 2 light quads), 4 views of 128x96, "
                      f"targets at 64 spp, {steps} Adam steps (lr 3e-3) at 8 spp, max_bounces 1, unbiased "
                      "estimator options; heights perturbed by N(0, 0.05), roughness by N(0, 0.1)",
           "full_configuration": "256x256 grid, 4 views of 1024x1024 at 256 spp, 200 steps at 64 spp, "
                                 "max_bounces 4: 268 M pixel samples fwd+bwd per step (not run)"}
    for arm, learned in (("plain", False), ("learned", True)):
        r = fit(FitConfig(steps=steps, learned=learned))
        out[arm] = {k: (round(v, 5) if isinstance(v, float) else v) for k, v in r.items()
                    if k in ("rmse_start", "rmse_final", "rmse_min", "time_to_goal_s", "steps_to_goal", "wall_s",
                             "samples_per_s")}
        h = r["history"]
        out[arm]["loss_first_last"] = [round(h[1]["loss"], 5), round(h[-1]["loss"], 5)]
        out[arm]["step_of_min"] = min(h, key=lambda x: x["rmse"])["step"]
    return out


# ---------------------------------------------------------------------------
# reference CPU renderer
# ---------------------------------------------------------------------------
def reference_step(wl, seed):
    """One step of the reference's own renderer: the forward call and the
    backward call (which renders again, render_pytorch.py:247-257).  Returns
    (forward seconds, backward seconds)."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    W, H = wl.resolution
    t0 = time.perf_counter()
    ref_runner.render_reference(wl, seed)
    t1 = time.perf_counter()
    ref_runner.render_reference(wl, seed, d_image=np.ones((H, W, 3), np.float32))
    return t1 - t0, time.perf_counter() - t1


def cpu_baseline():
    """The reference's own CPU path (oracle/_ref, -O3 -ffast-math, its thread pool
    on all host cores): two timed steps of the workload's scene at its reference
    sample size (10-30 s of CPU work) after a small page-in step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    if not ref_runner.reference_available() or WORKLOAD.get("no_reference"):
        return None
    reference_step(build_workload(REF_RES, spp=1), 0)  # page in, start the pool
    wl = build_workload(WORKLOAD["ref_res"], spp=WORKLOAD["ref_spp"])
    W, H = wl.resolution
    ts = [reference_step(wl, 1 + i) for i in range(2)]
    samples = W * H * wl.spp
    fwd = sum(t[0] for t in ts)
    total = sum(t[0] + t[1] for t in ts)
    return {"value": 2 * samples / total, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
            "forward": 2 * samples / fwd,
            "sample": f"2 steps of the workload's scene at {W}x{H}, {wl.spp} spp (forward call + backward call), "
                      f"{total:.1f} s"}


def run_reference(args):
    rank, _, world = dist_info()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    if not ref_runner.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
        return 0
    if WORKLOAD.get("no_reference"):
        print(json.dumps({"impl": "reference", "unavailable": WORKLOAD["no_reference"]}))
        return 0
    small = build_workload(REF_RES, spp=1)
    for i in range(args.warmup):  # warm-up on a 32x32 slice: pages in, starts the pool
        reference_step(small, 100 + i)
    wl = build_workload(WORKLOAD["ref_res"], spp=WORKLOAD["ref_spp"])
    W, H = wl.resolution
    ts = [reference_step(wl, i) for i in range(args.steps)]
    total = sum(a + b for a, b in ts)
    fwd = sum(a for a, _ in ts)
    samples = W * H * wl.spp
    value = samples * args.steps / total
    # linearity of the reference's time in samples: one step at twice the spp
    wl2 = build_workload(WORKLOAD["ref_res"], spp=2 * WORKLOAD["ref_spp"])
    a2, b2 = reference_step(wl2, 10_000)
    lin = {"spp": 2 * wl.spp, "value": 2 * samples / (a2 + b2), "ratio_to_value": 2 * samples / (a2 + b2) / value}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
            "impl": "reference", "forward": samples * args.steps / fwd,
            "config": {"workload": workload_label(), "resolution": list(WORKLOAD["resolution"]),
                       "spp": WORKLOAD["spp"], "max_bounces": wl.max_bounces, "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                             "sample": f"the same view at {W}x{H} x {wl.spp} spp per step (forward call + backward "
                                       f"call; per-sample work does not depend on the resolution), "
                                       f"{args.warmup} warm-up steps on a 32x32 slice"},
            "spp_linearity": lin,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def e2e_params(wl):
    """The parameters the end-to-end step differentiates: every shape's
    vertices except the lights', every material's roughness, the lights'
    intensities."""
    light_shapes = {l.shape_id for l in wl.lights}
    params = [s.vertices for i, s in enumerate(wl.shapes) if i not in light_shapes]
    params += [m.roughness for m in wl.materials]
    params += [l.intensity for l in wl.lights]
    return params


def run_b200(args):
    import numpy as np
    import torch
    from delta_ray_b200 import RenderFunction, _abi
    from delta_ray_b200.render_pytorch import Scene

    rank, local_rank, world = dist_info()
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)

    wl = build_workload()
    W, H = wl.resolution
    spp, B = wl.spp, wl.max_bounces  # spp: one step's batch
    samples = W * H * spp
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    scene = Scene(cam, mats, shps, lts, local_rank)
    d_img = torch.ones((H, W, 3), dtype=torch.float32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    from delta_ray_b200.distributed import average_gradients, rank_seed

    def step(seed, n_spp=spp):
        # each rank renders its own sample streams; one all-reduce combines the gradients
        s = rank_seed(seed, rank)
        scene.forward(W, H, n_spp, B, s)
        grad, _ = scene.backward(W, H, n_spp, B, s, d_img)
        if dist:
            average_gradients(grad)

    def timed(fn, count):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(count)]
        for k in range(count):
            flush.zero_()  # L2 flush between timed steps (outside the events)
            ev[k][0].record()
            fn(k)
            ev[k][1].record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev)

    def max_over_ranks(x):
        t = torch.tensor([x], device=dev)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for i in range(args.warmup):
        step(1000 + i)
    # per-kernel profile (untimed): kernel times and work counts for the roofline
    scene.set_profiling(True)
    scene.forward(W, H, spp, B, 7)
    stages = list(scene.last_timings())
    scene.backward(W, H, spp, B, 7, d_img)
    stages += scene.last_timings()
    # a streamed edge stage launches its kernels once per chunk of points:
    # each kernel's time is summed over the step, like the work counts
    launches_of = {}
    summed = {}
    for n, ms in stages:
        summed[n] = summed.get(n, 0.0) + ms
        launches_of[n] = launches_of.get(n, 0) + 1
    stages = list(summed.items())
    work = scene.last_work()
    scene.set_profiling(False)
    launches_per_step = 0
    scene.forward(W, H, spp, B, 8)
    launches_per_step += scene.launch_count()
    scene.backward(W, H, spp, B, 8, d_img)
    launches_per_step += scene.launch_count()

    clocks = ClockSampler(local_rank)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    total_ms = timed(step, args.steps)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    total_ms = max_over_ranks(total_ms)
    ms_per_step = total_ms / args.steps
    value = world * samples / (ms_per_step / 1e3)

    # forward only: the same batches, the forward call alone
    fwd_ms = max_over_ranks(timed(lambda k: scene.forward(W, H, spp, B, rank_seed(5000 + k, rank)), args.steps))
    forward_value = world * samples / (fwd_ms / args.steps / 1e3)

    # per-sample work does not depend on the batch: one step of twice the spp
    # (after an untimed one: the first call at a new size grows the queues)
    step(8999, 2 * spp)
    lin_ms = max_over_ranks(timed(lambda k: step(9000 + k, 2 * spp), 1))
    lin_value = world * 2 * samples / (lin_ms / 1e3)

    # end to end through the public API with host tensors: upload, scene build,
    # forward, loss read-back, backward, gradients back to the host
    wl_e2e = build_workload()
    params = e2e_params(wl_e2e)
    for x in params:
        x.requires_grad_(True)
    args_e2e = wl_e2e.serialize()
    h2d = sum(a.numel() * a.element_size() for a in args_e2e if torch.is_tensor(a))
    d2h = 4 + sum(x.numel() * x.element_size() for x in params)

    def e2e_step(seed):
        for x in params:
            x.grad = None
        img = RenderFunction.apply(rank_seed(seed, rank), *args_e2e)
        loss = img.sum()
        loss.item()
        loss.backward()
    for i in range(min(2, args.warmup)):
        e2e_step(500 + i)
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, 5))
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        e2e_step(600 + k)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps)
    e2e_value = world * samples / e2e_s

    # roofline of the dominant kernel (the longest one of a step, its
    # launches summed)
    peak, peak_kind = load_peaks()
    dom = max(stages, key=lambda s: s[1]) if stages else ("", 0.0)
    dom_bytes = kernel_bytes(dom[0], wl, work)
    achieved = dom_bytes / (dom[1] / 1e3) / 1e9 if dom[1] > 0 else 0.0
    prof = load_profile(dom[0])
    traffic = None
    if prof:  # DRAM bytes of the captured launch, scaled to this launch's units
        units = work["items"] if dom[0].startswith("k_edge") else samples
        traffic = int(prof["dram_bytes"] * units / max(1, prof["units"]))
    roofline = {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_step": dom_bytes,
                "l2": ({"hit_rate_pct": prof["l2_hit_pct"], "throughput_pct_of_peak": prof["l2_throughput_pct"],
                        "source": prof["source"]} if prof else None),
                "kernel_ms": {n: round(ms, 4) for n, ms in stages},
                "kernel_launches": launches_of,
                "kernel_model_gbs": {n: round(kernel_bytes(n, wl, work) / (ms / 1e3) / 1e9, 1)
                                     for n, ms in stages if ms > 0 and kernel_bytes(n, wl, work) > 0},
                "work": work}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
            "forward": forward_value,
            "config": {"workload": workload_label(), "resolution": [W, H], "spp": WORKLOAD["spp"],
                       "spp_per_step": spp, "max_bounces": B, "triangles": wl.num_triangles,
                       "parallelism": f"dp{world} (per-rank sample streams, gradient all-reduce)",
                       "l2": "flushed between steps (256 MB write)"},
            "spp_linearity": {"spp": 2 * spp, "value": lin_value, "ratio_to_value": lin_value / value},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches_per_step * args.steps, "roofline": roofline, "clocks": clk}
    if rank == 0 and world == 1 and not args.no_proposal:
        line["proposal"] = measure_proposal(dev, K=args.proposal_seeds, train_calls=args.proposal_train)
    if rank == 0 and world == 1 and not args.no_inverse and WORKLOAD_KEY == DEFAULT_WORKLOAD:
        try:
            line["inverse"] = measure_inverse(args.inverse_steps)
        except Exception as e:  # a report beside the headline, not part of it
            line["inverse"] = {"error": str(e)[:300]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline()
        except Exception as e:  # baseline is informative only
            line["cpu_baseline"] = {"unavailable": str(e)[:200]}
    if rank == 0:
        print(json.dumps(line))
    scene.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    global WORKLOAD, WORKLOAD_KEY
    args = parse()
    WORKLOAD = dict(WORKLOADS[args.workload])
    WORKLOAD_KEY = args.workload
    if args.res or args.step_spp:  # a smaller case of the same scene (profiling captures)
        if args.res:
            WORKLOAD["resolution"] = tuple(args.res)
        if args.step_spp:
            WORKLOAD["step_spp"] = WORKLOAD["spp"] = args.step_spp
        WORKLOAD_KEY = None  # no profile table, no inverse loop, no proposal report
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
