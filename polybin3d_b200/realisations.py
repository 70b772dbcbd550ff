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
import torch

from . import _native as nat

try:
    import torch.distributed as dist
except ImportError:  # pragma: no cover
    dist = None


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
        with torch.cuda.graph(self.graph):
            self.out = fn(self.seeds)
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
