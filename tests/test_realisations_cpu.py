"""Multi-rank host logic of the Monte Carlo Fisher (seed sharding + gather), on CPU with
world_size-2 `gloo` process groups: every rank must return the one-process mean bit for
bit, whatever the number of seeds per rank and the batch size."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from polybin3d_b200 import realisations

SHAPE = (6, 6)


def contrib(seeds):
    """Stand-in per-seed Fisher contribution: a seeded symmetric matrix."""
    out = []
    for s in seeds:
        a = np.random.default_rng(1000 + s).standard_normal(SHAPE)
        out.append(a + a.T)
    return np.stack(out)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, size, port, n_it, batch, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=timedelta(seconds=60))
    try:
        seen = []
        f = realisations.mc_mean(lambda s: (seen.extend(s), contrib(s))[1], n_it, SHAPE, "cpu", batch=batch)
        np.save(os.path.join(out_dir, "fish%d.npy" % rank), f.numpy())
        np.save(os.path.join(out_dir, "seeds%d.npy" % rank), np.asarray(seen, dtype=np.int64))
    finally:
        dist.destroy_process_group()


def _run(size, n_it, batch, tmp_path):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, size, port, n_it, batch, str(tmp_path))) for r in range(size)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    fish = [np.load(os.path.join(tmp_path, "fish%d.npy" % r)) for r in range(size)]
    seeds = [np.load(os.path.join(tmp_path, "seeds%d.npy" % r)) for r in range(size)]
    return fish, seeds


def serial_mean(n_it):
    """The one-process loop of compute_fisher: fish += f_seed / N_it in seed order."""
    fish = torch.zeros(SHAPE, dtype=torch.float64)
    for s in range(n_it):
        fish += torch.as_tensor(contrib([s])[0]) / n_it
    return fish.numpy()


def test_seed_partition():
    for n_it in (1, 2, 5, 8, 33):
        for size in (1, 2, 3, 8):
            parts = [realisations.seeds_of_rank(n_it, r, size) for r in range(size)]
            flat = sorted(s for p in parts for s in p)
            assert flat == list(range(n_it))
            assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


def test_one_process_matches_serial_loop():
    f = realisations.mc_mean(contrib, 7, SHAPE, "cpu", batch=3).numpy()
    assert np.array_equal(f, serial_mean(7))


@pytest.mark.parametrize("n_it,batch", [(5, 1), (8, 3)])
def test_two_ranks_gloo_bit_identical(tmp_path, n_it, batch):
    fish, seeds = _run(2, n_it, batch, tmp_path)
    ref = serial_mean(n_it)
    for r in range(2):
        assert np.array_equal(fish[r], ref)
        assert list(seeds[r]) == realisations.seeds_of_rank(n_it, r, 2)


def test_noise_pool_matches_the_reference_draw():
    """The spawned workers' draws equal np.random.seed(s); randn; randn (the reference's
    generate_data noise, base.py:315-332) for every seed, in order, through slot reuse."""
    import numpy as np
    import torch
    from polybin3d_b200 import realisations
    shape = (8, 8, 6)
    seeds = [3, 10000003, 7, 5, 20000001]
    pool = realisations.NoisePool(shape, workers=2)
    try:
        feed = pool.stream(seeds)
        re1, im1 = feed.take(2, torch.device("cpu"))
        re2, im2 = feed.take(3, torch.device("cpu"))
        re, im = torch.cat([re1, re2]), torch.cat([im1, im2])
        for i, s in enumerate(seeds):
            np.random.seed(s)
            r = np.random.randn(*shape)
            m = np.random.randn(*shape)
            assert np.array_equal(re[i].numpy(), r) and np.array_equal(im[i].numpy(), m), s
    finally:
        pool.close()
