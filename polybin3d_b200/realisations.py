"""Monte Carlo Fisher realisations sharded over ranks (one process per GPU).

`compute_fisher` is the mean of independent per-seed contributions over seeds 0..N_it-1
(PolyBin3D/pspec.py:553-569, bspec.py:678-693).  With a torch.distributed process group
of W ranks, rank r computes seeds r, r+W, r+2W, ...; the per-seed contributions are then
gathered to every rank and summed in seed order with the same arithmetic as the
one-process loop, so the mean does not depend on W: given the same per-seed contributions
it is bit-identical (the exchange is N_it x N_bins^2 FP64 values: 10.5 MB for 32
realisations of 203 bins).
Without an initialised process group (or with one rank) nothing is exchanged.
"""
import atexit
import gc
import multiprocessing
import os
from collections import deque
from concurrent.futures import ProcessPoolExecutor
from multiprocessing import shared_memory

import numpy as np
import torch

from . import _native as nat

try:
    import torch.distributed as dist
except ImportError:  # pragma: no cover
    dist = None


# --------------------------------------------------------------------------------------
# the reference's white noise, drawn ahead on host worker processes
# --------------------------------------------------------------------------------------
def _draw_reference_noise(shm_name, seed, shape):
    """Worker: np.random.seed(seed); randn(*shape) twice (PolyBin3D/base.py:315-316, 332),
    written into the shared-memory slot `shm_name` as [re, im]."""
    shm = shared_memory.SharedMemory(name=shm_name)
    try:
        out = np.ndarray((2,) + tuple(shape), dtype=np.float64, buffer=shm.buf)
        rs = np.random.RandomState(seed)  # the legacy global generator re-seeded with `seed`
        out[0] = rs.randn(*shape)
        out[1] = rs.randn(*shape)
        del out
    finally:
        shm.close()
    return seed


class NoisePool:
    """Spawned worker processes drawing the reference's MT19937 white noise into
    shared-memory slots.  The draw (two legacy Gaussian arrays per realisation) is
    single-threaded numpy in the reference and bounds a Monte Carlo loop fed with
    reference-identical noise; here W processes draw the realisations ahead of the one the
    device is working on.  Workers run numpy only (no CUDA), started with `spawn`."""

    def __init__(self, shape, workers=None):
        self.shape = tuple(int(n) for n in shape)
        self.workers = workers or max(1, min(16, (os.cpu_count() or 2) - 1))
        self.exe = ProcessPoolExecutor(max_workers=self.workers, mp_context=multiprocessing.get_context("spawn"))
        nbytes = 2 * int(np.prod(self.shape)) * 8
        self.slots = [shared_memory.SharedMemory(create=True, size=nbytes) for _ in range(2 * self.workers)]
        self.free = list(range(len(self.slots)))
        atexit.register(self.close)

    def close(self):
        if self.exe is not None:
            self.exe.shutdown(wait=True, cancel_futures=True)
            self.exe = None
        for s in self.slots:
            try:
                s.close()
                s.unlink()
            except FileNotFoundError:
                pass
        self.slots = []

    def stream(self, seeds):
        return NoiseFeed(self, seeds)


class NoiseFeed:
    """Noise for `seeds` in order: take(n, device) returns the next n draws as device FP64
    tensors (re, im) of shape (n, *grid); the freed slots go to the draws further ahead."""

    def __init__(self, pool, seeds):
        self.pool, self.todo, self.inflight = pool, deque(int(s) for s in seeds), deque()
        self._fill()

    def _fill(self):
        p = self.pool
        while self.todo and p.free:
            slot = p.free.pop()
            seed = self.todo.popleft()
            fut = p.exe.submit(_draw_reference_noise, p.slots[slot].name, seed, p.shape)
            self.inflight.append((seed, slot, fut))

    def take(self, n, device):
        p = self.pool
        re = torch.empty((n,) + p.shape, dtype=torch.float64, device=device)
        im = torch.empty_like(re)
        for i in range(n):
            if not self.inflight:
                raise RuntimeError("NoiseFeed: no draws left")
            seed, slot, fut = self.inflight.popleft()
            fut.result()
            view = np.ndarray((2,) + p.shape, dtype=np.float64, buffer=p.slots[slot].buf)
            re[i].copy_(torch.from_numpy(view[0]))  # pageable source: the copy is staged before returning
            im[i].copy_(torch.from_numpy(view[1]))
            del view
            p.free.append(slot)
            self._fill()
        return re, im

    def seeds_ahead(self):
        return [s for s, _, _ in self.inflight] + list(self.todo)


_POOLS = {}


def prefetch_pays(n_draws, shape):
    """Worker processes pay off once the draws add up to about a second of host time (their
    start-up costs a few seconds once per process)."""
    return n_draws >= 4 and n_draws * int(np.prod([int(n) for n in shape])) >= 8 * 128 ** 3


def noise_pool(shape):
    """The process-wide NoisePool for a grid shape (created on first use)."""
    key = tuple(int(n) for n in shape)
    pool = _POOLS.get(key)
    if pool is None:
        pool = NoisePool(key)
        _POOLS[key] = pool
    return pool


def world(group=None):
    """(rank, size) of `group`, or (0, 1) without an initialised process group."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def seeds_of_rank(N_it, rank, size):
    """Round-robin share of seeds 0..N_it-1 for `rank` of `size`."""
    return list(range(rank, N_it, size))


def _gather(local, size, group):
    """All ranks' (per, ...) blocks, rank-major, on local's device."""
    backend = dist.get_backend(group)
    comm = local if (backend == "nccl") == local.is_cuda else local.to("cuda" if backend == "nccl" else "cpu")
    parts = [torch.empty_like(comm) for _ in range(size)]
    dist.all_gather(parts, comm.contiguous(), group=group)
    return torch.cat(parts).to(local.device)


def mc_mean(contrib, N_it, shape, device, batch=1, group=None, progress=None):
    """Mean over seeds 0..N_it-1 of contrib(seeds) -> (len(seeds), *shape) FP64 tensors.

    `batch` seeds go to contrib per call; progress(seeds) is called on rank 0 before each
    call (the reference prints its progress line from there)."""
    rank, size = world(group)
    mine = seeds_of_rank(N_it, rank, size)
    per = (N_it + size - 1) // size
    shape = tuple(shape)
    local = torch.zeros((per,) + shape, dtype=torch.float64, device=device)
    for i0 in range(0, len(mine), batch):
        s = mine[i0:i0 + batch]
        if progress is not None and rank == 0:
            progress(s)
        local[i0:i0 + len(s)] = torch.as_tensor(contrib(s), dtype=torch.float64, device=device)
    if size > 1:
        every = _gather(local, size, group)
        index = [(s % size) * per + s // size for s in range(N_it)]
    else:
        every = local
        index = list(range(N_it))
    fish = torch.zeros(shape, dtype=torch.float64, device=device)
    for s in range(N_it):
        fish += every[index[s]] / N_it
    return fish


class CapturedBatch:
    """One CUDA graph of fn(seeds) -> tensor for a fixed batch of seeds.

    The first call runs fn once uncaptured (FFT plans, workspaces and cached device grids
    are created there), then captures it; every later batch writes its seeds into the
    captured seed tensor with one device arange and replays the graph, so a batch of
    realisations costs one graph launch and no host synchronisation.  The workspace
    buffers the graph uses are held for its lifetime.  `base` gets the FFT counts of
    each replay added, and the library's launch counter the launches of each replay."""

    def __init__(self, fn, batch, base):
        self.batch, self.base = batch, base
        self.seeds = torch.zeros(batch, dtype=torch.int64, device=base.device)
        fn(self.seeds)
        torch.cuda.synchronize(base.device)
        c0 = (base.n_FFTs_forward, base.n_FFTs_reverse, nat.LAUNCHES[0])
        self.graph = torch.cuda.CUDAGraph()
        # a finalizer that frees device memory (an unreferenced FFT plan, workspace or tensor
        # of earlier work) must not run inside the capture: a cudaFree there invalidates it.
        # Collect first, and keep the collector off while capturing.
        gc.collect()
        was_enabled = gc.isenabled()
        gc.disable()
        try:
            with torch.cuda.graph(self.graph):
                self.out = fn(self.seeds)
        finally:
            if was_enabled:
                gc.enable()
        self.delta = (base.n_FFTs_forward - c0[0], base.n_FFTs_reverse - c0[1], nat.LAUNCHES[0] - c0[2])
        self.keep = list(base.ws.bufs.values())

    def run(self, seeds):
        """Replay for an arithmetic progression of seeds (at most `batch`; a short batch is
        padded with the progression's continuation and those rows are dropped)."""
        seeds = [int(x) for x in seeds]
        step = seeds[1] - seeds[0] if len(seeds) > 1 else 1
        if any(seeds[i] != seeds[0] + i * step for i in range(len(seeds))) or len(seeds) > self.batch:
            raise ValueError("CapturedBatch.run needs an arithmetic progression of at most %d seeds" % self.batch)
        torch.arange(seeds[0], seeds[0] + step * self.batch, step, out=self.seeds)
        self.graph.replay()
        self.base.n_FFTs_forward += self.delta[0]
        self.base.n_FFTs_reverse += self.delta[1]
        nat.LAUNCHES[0] += self.delta[2]
        return self.out[:len(seeds)]
