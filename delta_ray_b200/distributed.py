"""Data-parallel rendering over several GPUs, one process per GPU.

Pixel samples are independent, so N ranks render the same scene with N
different random streams and the only exchange is the gradient: each rank's
flat gradient is an unbiased estimate, and their mean is the estimate of the
N-fold sample count (the reference has no multi-GPU path; its sum over
samples is delta_ray.cpp:1251-1459).  The collective is one all-reduce over
the flat gradient buffer per backward call (a few hundred floats for small
scenes, 12 * vertices + 256 bytes in general).
"""
_GOLDEN = 0x9E3779B97F4A7C15
_MASK = (1 << 64) - 1


def rank_seed(seed, rank):
    """The render seed of `rank` for the step seed `seed`: distinct per rank,
    so that the ranks' Philox streams are independent."""
    return (int(seed) * _GOLDEN + int(rank) * 0xD1B54A32D192ED03 + int(rank)) & _MASK


def average_gradients(flat, group=None):
    """Mean of the ranks' flat gradients, in place (one all-reduce)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return flat
    world = dist.get_world_size(group)
    if world == 1:
        return flat
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    flat.div_(world)
    return flat


def average_images(img, group=None):
    """Mean of the ranks' images, in place (forward of a sharded render)."""
    return average_gradients(img, group)


__all__ = ["rank_seed", "average_gradients", "average_images"]
