#!/usr/bin/env python
"""Forward+backward throughput of the B200 differentiable path tracer.

Workload: the soft-shadow scene (ground + 4-triangle blocker + area light),
512x512, 16 spp, max_bounces 1 -- one "step" renders the image and runs the
full backward (path adjoint, secondary edges, primary edges) against an
all-ones image adjoint.  Metric: pixel samples per second (fwd+bwd).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

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
# The headline workload is the soft-shadow scene (8 triangles, 512x512, 16 spp,
# max_bounces 1).  The heightfield scene (130,050 + 4 triangles, glossy, 2
# lights, max_bounces 3) runs at 160x120 and 4 spp: its shading points sample
# about 1,100 edges each under the reference's edge-tree rules, so the full
# 640x480 x 64 spp image would need 3e10 edge evaluations per backward call.
# ref_res, ref_spp: image size and samples per pixel of the reference CPU arm's
# steps (its time is linear in samples).
WORKLOADS = {
    "soft_shadow": dict(builder="soft_shadow", resolution=(512, 512), spp=16, max_bounces=1, scene_seed=0,
                        ref_res=(512, 512), ref_spp=16),
    "heightfield": dict(builder="heightfield", resolution=(160, 120), spp=4, max_bounces=3, scene_seed=0,
                        ref_res=(80, 60), ref_spp=1),
    # the same heightfield with GGX lobes; the reference has no GGX material, so
    # its arm reports this workload unavailable
    "heightfield_ggx": dict(builder="heightfield", resolution=(160, 120), spp=4, max_bounces=3, scene_seed=0,
                            ref_res=None, ref_spp=None, options={"microfacet": "ggx"},
                            no_reference="the reference's materials are Blinn-Phong only (no GGX lobe)"),
}
WORKLOAD = WORKLOADS["soft_shadow"]
# stages of the work model that run as several kernels
COMPOSITE_STAGES = {
    "k_primary_edges": ("k_primary_shade", "k_primary_grad"),
    "k_edge_traverse": ("k_edge_expand", "k_edge_tasks"),  # the two-stage walk of large edge trees
    "k_edge_eval": ("k_edge_line", "k_edge_rays", "k_edge_line_rays", "k_edge_shade"),
}
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
    p.add_argument("--workload", default="soft_shadow", choices=sorted(WORKLOADS))
    return p.parse_args()


def dist_info():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def build_workload(res=None, spp=None):
    from delta_ray_b200 import workloads
    w = WORKLOAD
    return workloads.BUILDERS[w["builder"]](seed=w["scene_seed"], resolution=res or w["resolution"],
                                            spp=spp or w["spp"], max_bounces=w["max_bounces"],
                                            **w.get("options", {}))


def workload_label():
    w = WORKLOAD
    opts = "".join(f" {k}={v}" for k, v in w.get("options", {}).items())
    return (f"{w['builder']} {w['resolution'][0]}x{w['resolution'][1]} {w['spp']}spp "
            f"max_bounces={w['max_bounces']}{opts} fwd+bwd")


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


def stage_bytes(stage, wl, counts):
    """Algorithmic bytes of one launch of a backward/forward stage."""
    W, H = wl.resolution
    spp, B = wl.spp, wl.max_bounces
    br = ray_bytes(wl.num_triangles)
    shade = 32 + 28  # path state read/write + material record per shading vertex
    n = W * H * spp
    points, items = counts
    rays_path = 1 + 2 * B  # upper bound: camera ray, then a shadow and a BSDF ray per bounce
    if stage in ("k_render_forward",):
        return n * (rays_path * br + B * shade) + W * H * 12
    if stage == "k_backward_paths":
        return n * (rays_path * br + B * shade) + W * H * 24 + points * 96
    if stage == "k_edge_traverse":
        return points * 96 + items * 20
    if stage == "k_edge_eval":
        # two straddling rays, two shadow rays of the emitter evaluations
        return items * (4 * br + 2 * shade + 96 + 20 + 12)
    if stage == "k_dp_propagate":
        return points * (96 + 36 + 12 * 3)
    if stage == "k_primary_edges":
        # two camera rays + two shaded paths per sample, plus edge/vertex reads
        return n * (2 * (1 + rays_path) * br + 2 * B * shade + 24 + 12)
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
    a reduced glossy heightfield (64 x 64-vertex grid, 7,938 triangles, 16
    patches, 80 x 60, 1 spp, B = 1) and a small one (10 x 10 grid, 162
    triangles, 96 x 72, 4 spp, B = 1, 3K seeds).  Per scene: K seeds of plain
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

    cases = [("heightfield 64x64-vertex grid (7,938 triangles), 80x60, 1 spp, max_bounces=1",
              lambda: workloads.heightfield(seed=0, resolution=(80, 60), spp=1, max_bounces=1, grid=64, patch=16), K),
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


def merge_stages(stages):
    """[(kernel, ms)] -> [(stage, ms)]: the kernels of a composite stage summed
    under its name (COMPOSITE_STAGES), other kernels kept, first-seen order."""
    parts_of = {k: name for name, parts in COMPOSITE_STAGES.items() for k in parts}
    merged = {}
    for name, ms in stages:
        key = parts_of.get(name, name)
        merged[key] = merged.get(key, 0.0) + ms
    return list(merged.items())


def load_traffic(stage):
    """DRAM bytes (read + write) per launch of `stage` from the committed ncu
    summary profiles/dram_traffic.txt ("<kernel> <bytes>" lines), if any; the
    edge-evaluation stage sums its wavefront's three kernels."""
    if WORKLOAD is not WORKLOADS["soft_shadow"]:
        return None  # the table was captured on the soft-shadow workload
    table = {}
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.txt")) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 2 and not line.startswith("#"):
                    table[parts[0]] = int(parts[1])
    except (OSError, ValueError):
        return None
    parts = COMPOSITE_STAGES.get(stage)
    if parts:  # the kernels of the stage that the captured build launched
        got = [table[k] for k in parts if k in table]
        return sum(got) if got else None
    return table.get(stage)


# ---------------------------------------------------------------------------
# reference CPU renderer
# ---------------------------------------------------------------------------
def reference_step(wl, seed):
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    W, H = wl.resolution
    t0 = time.perf_counter()
    ref_runner.render_reference(wl, seed)
    ref_runner.render_reference(wl, seed, d_image=np.ones((H, W, 3), np.float32))
    return time.perf_counter() - t0


def cpu_baseline():
    """The reference's own CPU path (oracle/_ref, -O3 -ffast-math, its thread pool
    on all host cores): two timed steps of the workload's scene at its reference
    size (about 10-20 s of CPU work on 16 cores) after a small page-in step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    if not ref_runner.reference_available() or WORKLOAD.get("no_reference"):
        return None
    reference_step(build_workload(REF_RES, spp=1), 0)  # page in, start the pool
    wl = build_workload(WORKLOAD["ref_res"], spp=WORKLOAD["ref_spp"])
    W, H = wl.resolution
    ts = [reference_step(wl, 1 + i) for i in range(2)]
    samples = W * H * wl.spp
    return {"value": 2 * samples / sum(ts), "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
            "sample": f"2 steps of the workload's scene at {W}x{H}, {wl.spp} spp (forward call + backward call), "
                      f"{sum(ts):.1f} s"}


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
    total = sum(ts)
    samples = W * H * wl.spp
    value = samples * args.steps / total
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
            "impl": "reference",
            "config": {"workload": workload_label(), "resolution": [W, H],
                       "spp": wl.spp,
                       "max_bounces": wl.max_bounces, "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                             "sample": f"{W}x{H} x {wl.spp} spp per step (forward call + backward call), "
                                       f"{args.warmup} warm-up steps on a 32x32 slice"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
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
    spp, B = wl.spp, wl.max_bounces
    samples = W * H * spp
    cam, mats, shps, lts = _abi.scene_dicts(wl.camera, wl.materials, wl.shapes, wl.lights)
    scene = Scene(cam, mats, shps, lts, local_rank)
    d_img = torch.ones((H, W, 3), dtype=torch.float32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    from delta_ray_b200.distributed import average_gradients, rank_seed

    def step(seed):
        # each rank renders its own sample streams; one all-reduce combines the gradients
        s = rank_seed(seed, rank)
        scene.forward(W, H, spp, B, s)
        grad, _ = scene.backward(W, H, spp, B, s, d_img)
        if dist:
            average_gradients(grad)

    for i in range(args.warmup):
        step(1000 + i)
    # per-stage profile (untimed): stage times and work counts for the roofline
    scene.set_profiling(True)
    scene.forward(W, H, spp, B, 7)
    stages = list(scene.last_timings())
    scene.backward(W, H, spp, B, 7, d_img)
    stages += scene.last_timings()
    counts = scene.last_counts()
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
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (outside the events)
        ev[k][0].record()
        step(k)
        ev[k][1].record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in ev)
    t = torch.tensor([total_ms], device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * samples / (ms_per_step / 1e3)

    # end to end through the public API with host tensors: upload, scene build,
    # forward, loss read-back, backward, gradients back to the host
    wl_e2e = build_workload()
    wl_e2e.shapes[1].vertices.requires_grad_(True)
    wl_e2e.lights[0].intensity.requires_grad_(True)
    wl_e2e.materials[0].diffuse_reflectance.requires_grad_(True)
    args_e2e = wl_e2e.serialize()
    h2d = sum(a.numel() * a.element_size() for a in args_e2e if torch.is_tensor(a))
    d2h = 4 + sum(x.numel() * x.element_size() for x in (wl_e2e.shapes[1].vertices, wl_e2e.lights[0].intensity,
                                                           wl_e2e.materials[0].diffuse_reflectance))

    def e2e_step(seed):
        for x in (wl_e2e.shapes[1].vertices, wl_e2e.lights[0].intensity, wl_e2e.materials[0].diffuse_reflectance):
            x.grad = None
        img = RenderFunction.apply(seed, *args_e2e)
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
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_t = torch.tensor([e2e_s], device=dev)
    if dist:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world * samples / float(e2e_t.item())

    # roofline of the dominant stage; a stage run as several kernels
    # (COMPOSITE_STAGES) counts as one
    peak, peak_kind = load_peaks()
    merged = merge_stages(stages)
    dom = max(merged, key=lambda s: s[1]) if merged else ("", 0.0)
    dom_bytes = stage_bytes(dom[0], wl, counts)
    achieved = dom_bytes / (dom[1] / 1e3) / 1e9 if dom[1] > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": dom[0], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": load_traffic(dom[0]),
                "algorithmic_bytes_per_launch": dom_bytes,
                "stage_ms": {n: round(ms, 4) for n, ms in stages},
                "points": counts[0], "edge_items": counts[1]}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
            "config": {"workload": workload_label(),
                       "resolution": [W, H], "spp": spp, "max_bounces": B, "triangles": wl.num_triangles,
                       "parallelism": f"dp{world} (per-rank sample streams, gradient all-reduce)", "l2": "flushed between steps (256 MB write)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches_per_step * args.steps, "roofline": roofline, "clocks": clk}
    if rank == 0 and world == 1 and not args.no_proposal:
        line["proposal"] = measure_proposal(dev, K=args.proposal_seeds, train_calls=args.proposal_train)
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
    global WORKLOAD
    args = parse()
    WORKLOAD = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
