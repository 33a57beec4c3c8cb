"""The inverse loop's smoothness prior (delta_ray_b200.inverse): its gradient
is that of the sum over neighbouring grid vertices of their squared height
difference (checked against autograd on the CPU)."""
import torch

from delta_ray_b200.inverse import FitConfig, HeightfieldFit


def test_smooth_grad_matches_autograd():
    f = object.__new__(HeightfieldFit)  # only the fields smooth_grad reads
    f.cfg = FitConfig(grid=7)
    h = torch.randn(49, dtype=torch.float64)
    f.heights = h.clone()
    x = h.clone().requires_grad_(True)
    g = x.reshape(7, 7)
    e = (g[:, 1:] - g[:, :-1]).pow(2).sum() + (g[1:, :] - g[:-1, :]).pow(2).sum()
    e.backward()
    assert torch.allclose(f.smooth_grad(), x.grad)
