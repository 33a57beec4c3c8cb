"""The learned proposal's network kernels (tcgen05, bf16 in, f32 accumulate)
against a float32 PyTorch reference of the same MLP.

The reference rounds what the kernels round (weights, inputs, hidden
activations, and in the backward pass the output gradient) to bf16 and keeps
everything else in f32, so the remaining differences are f32 summation order
and the rare activation whose bf16 rounding flips."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bf(t):
    return t.bfloat16().float()


def _reference(params, x, targets=None):
    from delta_ray_b200 import proposal
    leaf = params.detach().clone().requires_grad_(True)
    p = proposal.unflatten(leaf)

    class Round(torch.autograd.Function):  # bf16 forward, identity backward
        @staticmethod
        def forward(ctx, t):
            return _bf(t)

        @staticmethod
        def backward(ctx, g):
            return g

    h = _bf(x)
    for i in (1, 2, 3):
        h = Round.apply(torch.relu(h @ Round.apply(p[f"W{i}"]).T + p[f"b{i}"]))
    z = h @ Round.apply(p["W4"]).T + p["b4"]
    if targets is None:
        return z.detach()
    loss = -(targets * torch.log_softmax(z, 1)).sum() / targets.sum()
    loss.backward()
    return float(loss.detach()), leaf.grad


@pytest.mark.parametrize("n", [1, 300, 4096 + 17])
def test_forward_matches_float_reference(n):
    from delta_ray_b200 import proposal
    params = proposal.init_params(seed=n)
    x = torch.randn((n, 16), generator=torch.Generator().manual_seed(n))
    z = proposal.forward(params, x).cpu()
    ref = _reference(params, x)
    assert torch.isfinite(z).all()
    err = (z - ref).abs()
    assert err.max() <= 2e-2 * ref.abs().max() + 1e-3, float(err.max())
    assert err.mean() <= 2e-3 * ref.abs().max() + 1e-4, float(err.mean())


def test_gradient_matches_float_reference():
    from delta_ray_b200 import proposal
    n = 2048 + 64
    g = torch.Generator().manual_seed(3)
    params = proposal.init_params(seed=4)
    x = torch.randn((n, 16), generator=g)
    t = torch.rand((n, 32), generator=g) ** 4  # skewed targets
    t[::7] = 0.0                                 # rows without contribution
    loss, grad = proposal.gradient(params, x, t)
    ref_loss, ref_grad = _reference(params, x, t)
    grad = grad.cpu()
    assert np.isfinite(loss) and abs(loss - ref_loss) <= 1e-2 * abs(ref_loss)
    cos = float(grad @ ref_grad / (grad.norm() * ref_grad.norm()))
    assert cos > 0.999, cos
    assert float((grad - ref_grad).abs().max()) <= 3e-2 * float(ref_grad.abs().max())
    # every layer's block gets its share
    for name, v in proposal.unflatten(grad).items():
        r = proposal.unflatten(ref_grad)[name]
        assert float((v - r).norm()) <= 5e-2 * float(r.norm()) + 1e-7, name


def test_training_lowers_the_loss():
    """Adam on the network's gradient (a few hundred steps) fits targets that
    depend on the inputs."""
    from delta_ray_b200 import proposal
    g = torch.Generator().manual_seed(7)
    n = 4096
    x = torch.zeros((n, 16))
    x[:, :10] = torch.randn((n, 10), generator=g)
    slot = (x[:, 0] > 0).long() * 16 + (x[:, 1] > 0).long() * 8 + (x[:, 2] > 0).long()
    t = torch.zeros((n, 32))
    t[torch.arange(n), slot] = 1.0
    params = proposal.init_params(seed=8).cuda()
    m = torch.zeros_like(params)
    v = torch.zeros_like(params)
    first = None
    for step in range(1, 301):
        loss, grad = proposal.gradient(params, x, t)
        first = first if first is not None else loss
        m.mul_(0.9).add_(0.1 * grad)
        v.mul_(0.999).add_(0.001 * grad * grad)
        params -= 3e-3 * (m / (1 - 0.9 ** step)) / ((v / (1 - 0.999 ** step)).sqrt() + 1e-8)
    assert loss < 0.3 * first, (first, loss)
