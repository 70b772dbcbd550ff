"""Launch-shape autotuner for the kernels that have more than one good shape.

The first call of a shape (device, grid, map and pair counts, rows, precision) times every
candidate setting of pb_tuning_t (include/polybin3d_b200.h) with CUDA events on the current
stream, keeps the fastest and stores it in a JSON file, so later calls -- and later
processes -- set the winner before launching.  Tuned shapes:

* the tensor-core triplet contraction (from plain maps and from a tiled set): voxels per
  tile (plain maps: 128 / 64), staging ring depth, the barrier-wait form, accumulator sets
  (never the TMEM chain length, which changes the FP32 rounding);
* the k-bin reduction of many rows (>= 16): lane-per-row kernel (warps per block, blocks
  per SM) against the mode-tile kernel;
* routes that do the same work two ways (choose_route): the bispectrum's cubic sums from
  plain maps or from a tiled set (synthesis and contraction timed together).

Settings change launch shapes only; results agree to FP summation order.  Nothing is timed
while a CUDA graph is being captured (the default or the cached setting is used), and
PB_AUTOTUNE=0 turns tuning off.  The cache file is $PB_TUNING_CACHE, else
$XDG_CACHE_HOME/polybin3d_b200/tuning.json (~/.cache when XDG_CACHE_HOME is unset).
"""
import json
import os
import threading

import numpy as np
import torch

from . import _native as nat

# (launch shapes only: the TMEM chain length changes the FP32 rounding and stays fixed)
TC_CANDIDATES = [{}, {"tc_wait": 2}, {"tc_tile": 64}, {"tc_tile": 64, "tc_wait": 2}, {"tc_stages": 6},
                 {"tc_dsets": 1}]
# from a tiled map set (one contiguous copy per 128-voxel tile)
TC_TILED_CANDIDATES = [{}, {"tc_wait": 2}, {"tc_stages": 4}, {"tc_dsets": 1}, {"tc_wait": 2, "tc_dsets": 1}]
RED_CANDIDATES = [{}, {"red_method": 2}, {"red_method": 1, "red_warps": 2},
                  {"red_method": 1, "red_warps": 2, "red_waves": 16}, {"red_method": 1, "red_warps": 4, "red_waves": 4},
                  {"red_method": 1, "red_waves": 16}]


def cache_path():
    p = os.environ.get("PB_TUNING_CACHE")
    if p:
        return p
    root = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(root, "polybin3d_b200", "tuning.json")


def enabled():
    return os.environ.get("PB_AUTOTUNE", "1") != "0"


class Tuner:
    """Winners per shape key, persisted in a JSON file."""

    def __init__(self, path=None):
        self.path = path or cache_path()
        self.lock = threading.Lock()
        self.table = {}
        self.timings = {}
        try:
            with open(self.path) as f:
                self.table = json.load(f)
        except (OSError, ValueError):
            self.table = {}

    def _save(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            tmp = self.path + ".%d.tmp" % os.getpid()
            with open(tmp, "w") as f:
                json.dump(self.table, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except OSError:
            pass  # an unwritable cache only costs re-tuning in the next process

    def choose(self, key, candidates, run, reps=3):
        """The setting for `key`: the cached winner, or (on first use, outside graph capture)
        the fastest of `candidates` with run() timed under each; candidates[0] is the default."""
        with self.lock:
            hit = self.table.get(key)
        if hit is not None:
            return hit
        if not enabled() or torch.cuda.is_current_stream_capturing():
            return candidates[0]
        times = []
        for cfg in candidates:
            try:
                nat.set_tuning(cfg)
                run()  # warm-up (module load, first-launch set-up)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    run()
                e1.record()
                e1.synchronize()
                times.append(e0.elapsed_time(e1) / reps)
            except (NotImplementedError, ValueError, MemoryError):
                times.append(float("inf"))  # the shape does not fit this setting
            finally:
                nat.set_tuning(None)
        best = int(np.argmin(times))
        if not np.isfinite(times[best]):
            best = 0
        with self.lock:
            self.table[key] = dict(candidates[best])
            self.timings[key] = times
            self._save()
        return self.table[key]


    def choose_route(self, key, runs, reps=3):
        """The name of the fastest of `runs` (name -> callable doing the same work two ways),
        cached like a setting; the first name when tuning is off or a graph is being captured."""
        names = list(runs)
        with self.lock:
            hit = self.table.get(key)
        if hit is not None and hit.get("route") in runs:
            return hit["route"]
        if not enabled() or torch.cuda.is_current_stream_capturing():
            return names[0]
        times = []
        for name in names:
            try:
                runs[name]()  # warm-up (its own tuning, module load)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(reps):
                    runs[name]()
                e1.record()
                e1.synchronize()
                times.append(e0.elapsed_time(e1) / reps)
            except (NotImplementedError, ValueError, MemoryError):
                times.append(float("inf"))
        best = int(np.argmin(times))
        if not np.isfinite(times[best]):
            best = 0
        with self.lock:
            self.table[key] = {"route": names[best]}
            self.timings[key] = times
            self._save()
        return names[best]


_TUNER = None


def tuner():
    global _TUNER
    if _TUNER is None or _TUNER.path != cache_path():
        _TUNER = Tuner()
    return _TUNER


def device_tag(device):
    p = torch.cuda.get_device_properties(device)
    return "%s/%dsm" % (p.name.replace(" ", "_"), p.multi_processor_count)


class applied:
    """Context manager: pb_set_tuning(cfg) for the calls inside, defaults restored after."""

    def __init__(self, cfg):
        self.cfg = cfg

    def __enter__(self):
        if self.cfg:
            nat.set_tuning(self.cfg)
        return self

    def __exit__(self, *exc):
        if self.cfg:
            nat.set_tuning(None)


def contract(plan, A, B, C, out, ws, method, scale):
    """plan.contract with the tuned tensor-core launch shape for this shape."""
    if method != nat.PB_TRIPLET_TC:
        return plan.contract(A, B, C, out, ws, method=method, scale=scale)
    key = "tc|%s|%d|%d|%d|%d|%d" % (device_tag(A.device), A[0].numel(), A.shape[0], B.shape[0], C.shape[0],
                                    plan.n_pairs)
    cfg = tuner().choose(key, TC_CANDIDATES, lambda: plan.contract(A, B, C, out, ws, method=method, scale=scale))
    with applied(cfg):
        return plan.contract(A, B, C, out, ws, method=method, scale=scale)


def contract_tiled(plan, tiled, out, ws, scale):
    """plan.contract_tiled with the tuned launch shape for this shape."""
    key = "tct|%s|%d|%d|%d|%d" % (device_tag(tiled.data.device), tiled.n_vox, tiled.n_maps, tiled.n_factor,
                                  plan.n_pairs)
    cfg = tuner().choose(key, TC_TILED_CANDIDATES, lambda: plan.contract_tiled(tiled, out, ws, scale=scale))
    with applied(cfg):
        return plan.contract_tiled(tiled, out, ws, scale=scale)


def bin_reduce(grid, precision, mode, a, b, n_rows, edges, ells, scale, out, ws, accumulate=False, row_stride=0):
    """nat.bin_reduce with the tuned kernel for many rows (candidates are timed on a scratch
    output, so an accumulating call is not applied more than once)."""
    if n_rows < 16:
        return nat.bin_reduce(grid, precision, mode, a, b, n_rows, edges, ells, scale, out, ws, accumulate,
                              row_stride)
    nk = len(edges) - 1
    n_ell = len(np.asarray(ells).reshape(-1)) // 2
    dev = out.device
    key = "red|%s|%d,%d,%d|%d|%d|%d|%d|%d" % (device_tag(dev), grid.n[0], grid.n[1], grid.n[2], n_rows, nk, n_ell,
                                              precision, mode)
    scratch = None

    def run():
        nonlocal scratch
        if scratch is None:
            scratch = torch.empty_like(out)
        nat.bin_reduce(grid, precision, mode, a, b, n_rows, edges, ells, scale, scratch, ws, False, row_stride)

    cfg = tuner().choose(key, RED_CANDIDATES, run)
    with applied(cfg):
        return nat.bin_reduce(grid, precision, mode, a, b, n_rows, edges, ells, scale, out, ws, accumulate,
                              row_stride)
