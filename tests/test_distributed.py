"""Multi-rank host logic on CPU (gloo, world size 2): per-rank seeds and the
gradient all-reduce of a data-parallel render.  The per-rank gradients are the
oracle's (Philox mode, the product's streams), so the test also checks that
the mean over ranks is the mean of independent renders."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import oracle
        from delta_ray_b200 import workloads
        from delta_ray_b200.distributed import average_gradients, rank_seed
        wl = workloads.single_triangle(1, (16, 16), 2, 1)
        seed = rank_seed(9, rank)
        o = oracle.oracle_render(wl, seed, np.ones((16, 16, 3), np.float32), rng_mode=oracle.PHILOX, threads=1)
        flat = torch.from_numpy(np.ascontiguousarray(o["grad"], np.float32))
        np.save(os.path.join(out_dir, f"grad{rank}.npy"), flat.numpy())
        np.save(os.path.join(out_dir, f"seed{rank}.npy"), np.array([seed], np.uint64))
        average_gradients(flat)
        np.save(os.path.join(out_dir, f"mean{rank}.npy"), flat.numpy())
    finally:
        dist.destroy_process_group()


def test_rank_seeds_are_distinct():
    from delta_ray_b200.distributed import rank_seed
    seeds = {rank_seed(s, r) for s in range(64) for r in range(8)}
    assert len(seeds) == 64 * 8
    assert all(0 <= x < 2 ** 64 for x in seeds)


def test_gradient_allreduce_two_ranks(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    g0, g1 = (np.load(tmp_path / f"grad{r}.npy") for r in range(2))
    s0, s1 = (int(np.load(tmp_path / f"seed{r}.npy")[0]) for r in range(2))
    assert s0 != s1
    assert not np.array_equal(g0, g1)  # independent sample streams
    want = (g0.astype(np.float64) + g1) / 2
    for r in range(2):
        m = np.load(tmp_path / f"mean{r}.npy")
        assert np.allclose(m, want, rtol=1e-6, atol=1e-7)
