"""Inverse rendering of the glossy heightfield: fit a height grid and the
per-patch roughness to target images of several views.

The loop restates the reference's optimisation demos (test/test_shadow.py:
66-83, Adam on scene parameters against an image L2 loss;
heightfield_gan.py:247-266 for saving state) on the B200 path: one device
scene per view, updated in place between steps (dr_scene_update: LBVH refit,
edge topology kept, edge trees and primary samplers rebuilt on the GPU), a
forward and a backward call per view per step, the flat gradient mapped back
to the grid heights and the roughness, and torch's Adam.  With the learned
edge proposal on, every view's scene trains its proposal network online from
the backward calls.  Checkpoints (torch.save) hold the parameters, the Adam
state, the step and every view's proposal network; a fit resumes from one.

Full configuration: the heightfield of bench.py's default workload
(256 x 256 grid) with targets at 1024 x 1024, 256 spp from 4 views, 200 Adam
steps at 64 spp, max_bounces 4.  A step of that is 4 x 1024^2 x 64 = 268 M
pixel samples forward and backward; `FitConfig` defaults to a reduced
setting (64 x 64 grid, 128 x 96 views) that runs in minutes.

    python -m delta_ray_b200.inverse [--steps 200] [--learned] [--grid 64] ...
"""
import argparse
import json
import math
import os
import time
from dataclasses import asdict, dataclass, field

import numpy as np
import torch

from . import _abi, workloads
from .render_pytorch import RenderOptions, Scene


@dataclass
class FitConfig:
    grid: int = 64                # heightfield vertices per side
    patch: int = 16               # vertices per roughness patch side
    resolution: tuple = (128, 96)
    views: int = 4
    target_spp: int = 64
    spp: int = 8                  # per view per step
    # direct lighting: with more bounces the reference's edge estimator gives
    # the heights a gradient along a common height shift that finite
    # differences of the loss do not show, and the fit drifts along it
    max_bounces: int = 1
    steps: int = 200
    lr: float = 3e-3
    height_noise: float = 0.05    # initial perturbation of the heights (std)
    roughness_noise: float = 0.1  # initial perturbation of the roughness (std)
    rmse_goal: float = 0.01
    common_seeds: bool = False    # common random numbers: targets at `spp` with each view's seed, reused every step
    # unbiased estimators (every sampled edge's position derivative summed,
    # the sampling pdf held constant, lobe mixture weights for edge samples,
    # sub-pixel samples over the whole pixel); False: the reference's
    unbiased: bool = True
    # weight of a smoothness prior on the heights: smooth * the sum over
    # neighbouring grid vertices of their squared height difference, added to
    # the image loss (0: none)
    smooth: float = 0.0
    learned: bool = False         # train and use the learned edge proposal
    proposal_mix: float = 0.8
    seed: int = 0
    checkpoint_dir: str = ""      # save a checkpoint every checkpoint_every steps when set
    checkpoint_every: int = 50
    device: int = 0


def view_cameras(n, resolution, radius=10.5, height=7.0):
    """n cameras on a circle around the heightfield, looking at its centre."""
    cams = []
    for k in range(n):
        a = 2 * math.pi * k / n
        eye = [radius * math.sin(a), height, -radius * math.cos(a)]
        cams.append(workloads._camera(eye, [0.0, 0.0, 0.0], [0.0, 1.0, 0.0], 45.0, list(resolution)))
    return cams


class HeightfieldFit:
    """State of one fit: the target scene, the parameters and the per-view
    device scenes."""

    def __init__(self, cfg: FitConfig):
        self.cfg = cfg
        self.dev = torch.device("cuda", cfg.device)
        wl = workloads.heightfield(seed=cfg.seed, resolution=cfg.resolution, spp=cfg.spp,
                                   max_bounces=cfg.max_bounces, grid=cfg.grid, patch=cfg.patch)
        self.wl = wl
        self.n_patch = len(wl.meta["patch_grid_index"])
        self.true_heights = torch.from_numpy(wl.meta["heights"]).reshape(-1)
        self.true_rough = torch.stack([wl.materials[i].roughness.reshape(()) for i in range(self.n_patch)])
        self.index = [torch.from_numpy(np.asarray(ix, np.int64)) for ix in wl.meta["patch_grid_index"]]
        self.xz = [wl.shapes[i].vertices[:, [0, 2]].clone() for i in range(self.n_patch)]
        self.cams = view_cameras(cfg.views, cfg.resolution)
        rng = np.random.default_rng(cfg.seed + 1)
        h0 = self.true_heights + torch.from_numpy(rng.normal(0, cfg.height_noise, self.true_heights.shape)
                                                  .astype(np.float32))
        r0 = (self.true_rough + torch.from_numpy(rng.normal(0, cfg.roughness_noise, self.n_patch)
                                                 .astype(np.float32))).clamp(0.02, 1.0)
        self.heights = h0.clone().requires_grad_(True)
        self.rough = r0.clone().requires_grad_(True)
        self.opt = torch.optim.Adam([self.heights, self.rough], lr=cfg.lr)
        self.step = 0
        self.scenes = None
        self.targets = None

    # -- scene construction ------------------------------------------------
    def _scene_lists(self, heights, rough):
        """Materials and shapes of the heightfield with these parameters."""
        wl = self.wl
        shapes = []
        for i, s in enumerate(wl.shapes):
            if i < self.n_patch:
                y = heights.detach()[self.index[i]].reshape(-1, 1)
                v = torch.cat([self.xz[i][:, :1], y, self.xz[i][:, 1:]], 1).contiguous()
                shapes.append(workloads.Shape(v, s.indices, s.uvs, s.normals, s.mat_id))
            else:
                shapes.append(s)
        mats = []
        for i, m in enumerate(wl.materials):
            if i < self.n_patch:
                mats.append(workloads.Material(m.diffuse_reflectance, m.specular_reflectance,
                                               rough.detach()[i].reshape(1).contiguous(),
                                               two_sided=m.two_sided,
                                               microfacet=("blinn_phong", "ggx")[int(m.microfacet)]))
            else:
                mats.append(m)
        return mats, shapes

    def _dicts(self, cam, mats, shapes):
        return _abi.scene_dicts(cam, mats, shapes, self.wl.lights)

    def options(self, backward=False):
        """Render options of the fit's forward or backward calls (the learned
        proposal only draws the backward call's edges)."""
        learned = backward and self.cfg.learned
        if not self.cfg.unbiased:
            return RenderOptions(learned_proposal=learned)
        return RenderOptions(dp_mode=_abi.DR_DP_SUM, detached_pdf=True, edge_lobe_mis=True, full_pixel_jitter=True,
                             learned_proposal=learned)

    def view_seed(self, k):
        """Seed of view k at the current step (the same at every step with
        common_seeds, and then also the target's)."""
        return 777 + k if self.cfg.common_seeds else 100_000 * (k + 1) + self.step

    def render_targets(self):
        """Target images of every view (forward only): target_spp samples, or
        with common_seeds the fit's spp on the fit's own sample streams."""
        mats, shapes = self._scene_lists(self.true_heights, self.true_rough)
        self.targets = []
        W, H = self.cfg.resolution
        spp = self.cfg.spp if self.cfg.common_seeds else self.cfg.target_spp
        for k, cam in enumerate(self.cams):
            c, m, s, l = self._dicts(cam, mats, shapes)
            sc = Scene(c, m, s, l, self.cfg.device)
            try:
                self.targets.append(sc.forward(W, H, spp, self.cfg.max_bounces, 777 + k, self.options()).clone())
            finally:
                sc.close()
        return self.targets

    def _ensure_scenes(self, mats, shapes):
        if self.scenes is None:
            self.scenes = []
            for cam in self.cams:
                c, m, s, l = self._dicts(cam, mats, shapes)
                sc = Scene(c, m, s, l, self.cfg.device)
                if self.cfg.learned:
                    sc.set_proposal(train=True, mix=self.cfg.proposal_mix, learning_rate=3e-3, train_points=16384)
                self.scenes.append(sc)
        else:
            for cam, sc in zip(self.cams, self.scenes):
                c, m, s, l = self._dicts(cam, mats, shapes)
                sc.update(c, m, s, l)

    # -- one Adam step -------------------------------------------------------
    def rmse(self):
        d = torch.cat([self.heights.detach() - self.true_heights, self.rough.detach() - self.true_rough])
        return float(d.pow(2).mean().sqrt())

    def adam_step(self):
        cfg = self.cfg
        W, H = cfg.resolution
        mats, shapes = self._scene_lists(self.heights, self.rough)
        self._ensure_scenes(mats, shapes)
        opts, fwd_opts = self.options(backward=True), self.options()
        g_h = torch.zeros_like(self.true_heights)
        g_r = torch.zeros(self.n_patch)
        loss = 0.0
        for k, sc in enumerate(self.scenes):
            seed = self.view_seed(k)
            img = sc.forward(W, H, cfg.spp, cfg.max_bounces, seed, fwd_opts)
            diff = img - self.targets[k]
            loss += float(diff.pow(2).mean())
            d_img = (2.0 / diff.numel()) * diff
            grad, _ = sc.backward(W, H, cfg.spp, cfg.max_bounces, seed, d_img.contiguous(), opts)
            parts = sc.sd.split_grad(grad.cpu(), sc.materials, sc.shapes)
            for i in range(self.n_patch):
                g_h.index_add_(0, self.index[i], parts["d_vertices"][i][:, 1])
                g_r[i] += parts["d_roughness"][i].reshape(())
        if cfg.smooth > 0.0:
            g_h += cfg.smooth * self.smooth_grad()
        self.opt.zero_grad()
        self.heights.grad = g_h
        self.rough.grad = g_r
        self.opt.step()
        with torch.no_grad():
            self.rough.clamp_(0.02, 1.0)
        self.step += 1
        return loss

    def smooth_grad(self):
        """Gradient of the sum over neighbouring grid vertices of their
        squared height difference."""
        g = self.cfg.grid
        h = self.heights.detach().reshape(g, g)
        out = torch.zeros_like(h)
        dx = h[:, 1:] - h[:, :-1]
        dz = h[1:, :] - h[:-1, :]
        out[:, 1:] += 2 * dx
        out[:, :-1] -= 2 * dx
        out[1:, :] += 2 * dz
        out[:-1, :] -= 2 * dz
        return out.reshape(-1)

    # -- checkpoints ---------------------------------------------------------
    def state_dict(self):
        st = {"step": self.step, "heights": self.heights.detach().clone(), "rough": self.rough.detach().clone(),
              "adam": self.opt.state_dict(), "config": asdict(self.cfg)}
        if self.cfg.learned and self.scenes:
            st["proposal"] = [sc.proposal_state()[0] for sc in self.scenes]
        return st

    def save(self, path):
        torch.save(self.state_dict(), path)

    def load(self, path):
        st = torch.load(path, weights_only=False)
        with torch.no_grad():
            self.heights.copy_(st["heights"])
            self.rough.copy_(st["rough"])
        self.opt.load_state_dict(st["adam"])
        self.step = int(st["step"])
        if "proposal" in st:
            mats, shapes = self._scene_lists(self.heights, self.rough)
            self._ensure_scenes(mats, shapes)
            for sc, p in zip(self.scenes, st["proposal"]):
                sc.set_proposal(train=True, mix=self.cfg.proposal_mix, learning_rate=3e-3, train_points=16384,
                                params=p)

    def close(self):
        for sc in self.scenes or []:
            sc.close()
        self.scenes = None


def fit(cfg: FitConfig, log=None):
    """Runs the fit; returns the history and the time to reach the RMSE goal."""
    f = HeightfieldFit(cfg)
    try:
        f.render_targets()
        torch.cuda.synchronize()
        hist = [{"step": 0, "rmse": f.rmse(), "loss": None, "s": 0.0}]
        t_goal = None
        t0 = time.perf_counter()
        for _ in range(cfg.steps):
            loss = f.adam_step()
            torch.cuda.synchronize()
            t = time.perf_counter() - t0
            r = f.rmse()
            hist.append({"step": f.step, "rmse": r, "loss": loss, "s": t})
            if t_goal is None and r <= cfg.rmse_goal:
                t_goal = t
            if cfg.checkpoint_dir and f.step % cfg.checkpoint_every == 0:
                os.makedirs(cfg.checkpoint_dir, exist_ok=True)
                f.save(os.path.join(cfg.checkpoint_dir, f"step{f.step:05d}.pt"))
            if log:
                log(hist[-1])
        samples = cfg.steps * cfg.views * cfg.resolution[0] * cfg.resolution[1] * cfg.spp
        return {"config": asdict(cfg), "rmse_start": hist[0]["rmse"], "rmse_final": hist[-1]["rmse"],
                "rmse_min": min(h["rmse"] for h in hist), "time_to_goal_s": t_goal,
                "steps_to_goal": next((h["step"] for h in hist if h["rmse"] <= cfg.rmse_goal), None),
                "wall_s": hist[-1]["s"], "samples_per_s": samples / max(1e-9, hist[-1]["s"]),
                "history": hist}
    finally:
        f.close()


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    cfg = FitConfig()
    for k, v in asdict(cfg).items():
        if isinstance(v, bool):
            p.add_argument("--" + k.replace("_", "-"), action="store_true", default=v)
        elif isinstance(v, tuple):
            p.add_argument("--" + k.replace("_", "-"), type=int, nargs=len(v), default=list(v))
        else:
            p.add_argument("--" + k.replace("_", "-"), type=type(v), default=v)
    a = p.parse_args(argv)
    kw = {k: (tuple(getattr(a, k)) if isinstance(v, tuple) else getattr(a, k)) for k, v in asdict(cfg).items()}
    res = fit(FitConfig(**kw))
    res.pop("history")
    print(json.dumps(res))


if __name__ == "__main__":
    main()
