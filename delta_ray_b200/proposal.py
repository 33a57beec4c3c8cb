"""The learned edge proposal's network (a project addition; the reference
samples edges by its edge-tree importance alone).

A 10 -> 64 -> 64 -> 64 -> 32 MLP with ReLU hidden layers and a softmax
output, run and trained by the library's tensor-core kernels in bf16 with f32
accumulation.  Its inputs are a shading point's position (normalised to the
scene bounds), shading normal, roughness and incoming direction; its 32
outputs are probabilities over directions from the point (4 bands of
cos(theta) times 8 azimuth sectors in the shading frame).  Edge sampling
weights each edge-tree child's importance by the probability of the
direction towards it, so the network can learn what the importance bound
does not model, such as occlusion.

``init_params``  a fresh parameter vector (PyTorch nn.Linear initialisation)
``forward``      logits of rows x [n, 16] (inputs 10..15 zero for the proposal)
``gradient``     (loss, gradient) of sum_rows sum_s -t[s] log softmax(z)[s] / sum(t)
"""
import ctypes as C

import torch

from . import _lib

IN, HIDDEN, OUT, FEATURES = 16, 64, 32, 10
SHAPES = [("W1", (64, 16)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)), ("W3", (64, 64)), ("b3", (64,)),
          ("W4", (32, 64)), ("b4", (32,))]


def param_count():
    return int(_lib.lib().dr_mlp_param_count())


def unflatten(params):
    """Dict name -> view of the flat parameter vector."""
    out, o = {}, 0
    for name, shape in SHAPES:
        n = 1
        for d in shape:
            n *= d
        out[name] = params[o:o + n].view(*shape)
        o += n
    return out


def init_params(seed=0, device="cpu"):
    """nn.Linear's default initialisation: U(-1/sqrt(fan_in), 1/sqrt(fan_in)),
    with W1's fan-in the 10 real features."""
    g = torch.Generator().manual_seed(int(seed))
    parts = []
    for name, shape in SHAPES:
        fan_in = FEATURES if name in ("W1", "b1") else shape[-1] if name.startswith("W") else HIDDEN
        bound = 1.0 / fan_in ** 0.5
        parts.append((torch.rand(shape, generator=g) * 2 - 1).mul_(bound).reshape(-1))
    p = torch.cat(parts)
    assert p.numel() == param_count()
    return p.to(device)


def _dev(t):
    return torch.as_tensor(t, dtype=torch.float32).cuda().contiguous()


def forward(params, x):
    """Logits [n, 32] (CUDA) of rows x [n, 16]."""
    params, x = _dev(params), _dev(x)
    n = x.shape[0]
    logits = torch.empty((n, OUT), dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib().dr_mlp_forward(C.c_void_p(params.data_ptr()), C.c_void_p(x.data_ptr()), n,
                                         C.c_void_p(logits.data_ptr()), None))
    return logits


def gradient(params, x, targets):
    """(loss, gradient [param_count()]) of the weighted cross-entropy."""
    params, x, targets = _dev(params), _dev(x), _dev(targets)
    grads = torch.empty(param_count(), dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib().dr_mlp_gradient(C.c_void_p(params.data_ptr()), C.c_void_p(x.data_ptr()),
                                          C.c_void_p(targets.data_ptr()), x.shape[0], C.c_void_p(grads.data_ptr()),
                                          C.c_void_p(loss.data_ptr()), None))
    return float(loss.item()), grads
