"""Benchmark: Bk_ideal fields/s at 256^3 (16 bins, lmax=2, TSC, mixed precision).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--contraction auto|tc|simt]
                    [--workload ...] [--route auto|plain|tiled]

One step = one float32 lognormal field through BSpec.Bk_ideal: r2c, the synthesis of the
32 bin-filtered maps (Theta_b L_l / W_TSC) on the dealiased 192^3 grid (pb_shell_synth:
band-limited filter and inverse transform as pruned passes), the tensor-core triplet
contraction over 888 bin triplets, and the inverse ideal Fisher (cached, as the reference
caches it).  The maps and the contraction take the route Bk_ideal takes: plain maps or a
tiled map set, whichever the autotuner timed faster for this shape (--route pins one).  `value` times that on device-resident fields; `e2e` times the
public call Bk_ideal(field) on pinned host fields, H2D copy and result readback included.
Under torchrun every rank runs independent fields (replicas: a 256^3 field does not
shard), timing is the max over ranks and `value` counts all ranks' fields.

The same line carries the metric's second half under "fisher": Monte Carlo Fisher
realisations/s at 128^3 for PSpec (lmax=4, 60 bins) and BSpec (lmax=0, 203 bins) on the
200-hole shell-sector mask -- device noise in captured graphs as `value`, the
reference-identical MT19937 noise (drawn by host worker processes) as `e2e` -- each with
its HBM fraction and CPU baseline.  --workload bk256 runs the Bk line alone,
fisher_pk128 | fisher_bk128 one Fisher workload, bk512grad the 512^3 forward + gradient.

--impl reference times the reference's own CPU implementation of the same step on the
host cores: its compiled Cython assemble_b3 (oracle/_ref, built from the reference's
utils.pyx) with FP64 scipy FFTs and the filter loop of bspec.py:912-956, on a bounded
sample of each field's triplets when a whole field would take too long.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

N, L, LMAX, NK = 256, 2000.0, 2, 16
EDGES = np.linspace(2 * np.pi / L, 0.2, NK + 1)
METRIC = "Bk fields/s at 256^3 (16 bins, lmax=2, TSC, mixed precision)"
WORKLOAD = "Bk_ideal 256^3 box 2000 Mpc/h, TSC, lmax=2, 16 linear bins 2pi/2000..0.2, 888 triangle bins"
# DRAM bytes (read + write) of one tensor-core contraction launch of this workload,
# dram__bytes_read.sum + dram__bytes_write.sum from one ncu capture each: from a tiled set of 32
# maps (16 pair factors) on the 192^3 grid (1,358,954,496 algorithmic bytes), and from the
# 32 plain FP32 maps (905,969,664 algorithmic bytes)
TC_TRAFFIC_TILED = 1_359_059_000 + 5_238_784
TC_TRAFFIC_PLAIN = 906_144_256 + 3_914_752


FISHER = {
    # Pk_unwindowed + PSpec.compute_fisher: 128^3, box 1500, lmax=4, 20 bins to 0.25, shell-sector mask
    "fisher_pk128": dict(N=128, L=1500.0, lmax=4, edges=np.linspace(2 * np.pi / 1500.0, 0.25, 21), batch=8,
                         metric="Pk Fisher MC sims/s at 128^3 (60 bins, lmax=4, masked)",
                         workload="PSpec.compute_fisher 128^3 box 1500 Mpc/h, lmax=4, 20 linear bins 2pi/1500..0.25, "
                                  "shell-sector mask with 200 holes"),
    # Bk_unwindowed + BSpec.compute_fisher: 128^3, box 1500, lmax=0, 12 bins to 0.2, same mask
    "fisher_bk128": dict(N=128, L=1500.0, lmax=0, edges=np.linspace(2 * np.pi / 1500.0, 0.2, 13), batch=1,
                         metric="Bk Fisher MC sims/s at 128^3 (203 bins, lmax=0, masked)",
                         workload="BSpec.compute_fisher 128^3 box 1500 Mpc/h, lmax=0, 12 linear bins 2pi/1500..0.2, "
                                  "shell-sector mask with 200 holes"),
}


FISHER_STEPS = 4  # batches per Monte Carlo Fisher record of the default run

# Bk_ideal + its gradient at 512^3: 24 bins to 0.35, lmax=2, TSC, mixed precision, streamed fields
BK512 = dict(N=512, L=4000.0, lmax=2, edges=np.linspace(2 * np.pi / 4000.0, 0.35, 25),
             metric="Bk_ideal + dBk/ddelta fields/s at 512^3 (24 bins, lmax=2, TSC, mixed precision)",
             workload="Bk_ideal and its vector-Jacobian product dBk/ddelta^T v, 512^3 box 4000 Mpc/h, TSC, lmax=2, "
                      "24 linear bins 2pi/4000..0.35, 2756 triangle bins; g-maps recomputed in the backward")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=None)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    # headline (default): the 256^3 Bk line with the Monte Carlo Fisher records inside it;
    # bk256: the Bk line alone; fisher_*: one Fisher workload alone; bk512grad: 512^3 forward + gradient
    p.add_argument("--workload", default="headline", choices=["headline", "bk256", "bk512grad"] + sorted(FISHER))
    p.add_argument("--contraction", default="auto", choices=["auto", "tc", "simt"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    # the bispectrum's cubic-sum route: auto (the autotuner's choice, as Bk_ideal uses it), or one
    # of the two pinned (for profiling a kernel of that route)
    p.add_argument("--route", default="auto", choices=["auto", "plain", "tiled"])
    a = p.parse_args()
    if a.steps is None:
        a.steps = {"headline": 50, "bk256": 50, "bk512grad": 16}.get(a.workload, 6)
    return a


def fisher_mask(N, L):
    """Shell 250 < r < 700 Mpc/h about the box centre, octant x,y,z > 0, 200 seeded holes of
    radius 5-20 Mpc/h (float32)."""
    from polybin3d_b200 import synthetic
    return synthetic.shell_mask(N, L, r_in=250.0, r_out=700.0, n_holes=200, hole_r=(5.0, 20.0), hole_box=700.0,
                                seed=0)


class Clocks:
    """Sample nvidia-smi SM clocks and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 6:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[2 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_reference_step(bs, frac, field, nthreads, ref_utils):
    """One (sampled) field of the reference's numerator on the host, FP64.
    Filtering and FFTs follow bspec.py:912-956; the cubic sum is the reference's compiled
    assemble_b3 when oracle/_ref is built, else the oracle's C loop."""
    from oracle import polybin_oracle as O
    x = bs.weighted_data(field, "ideal")
    g = bs.g_maps(x)
    ab = bs.all_bins
    n = int(round(frac * len(ab)))
    if n == 0:
        return None
    sub = np.ascontiguousarray(ab[:n])
    if ref_utils is not None:
        B3 = ref_utils.assemble_b3(np.ascontiguousarray(g), sub, nthreads)
    else:
        flat = g.reshape(bs.Nl * bs.Nk_squeeze, -1)
        B3 = O.triplet_sum(flat, flat, flat, bs.triplet_index()[:n], nthreads)
    return B3


def load_ref_utils():
    import importlib.util
    d = os.path.join(REPO, "oracle", "_ref")
    if not os.path.isdir(d):
        return None
    for f in os.listdir(d):
        if f.startswith("pb_ref_utils") and f.endswith(".so"):
            spec = importlib.util.spec_from_file_location("pb_ref_utils", os.path.join(d, f))
            m = importlib.util.module_from_spec(spec)
            try:
                spec.loader.exec_module(m)
                return m
            except Exception:
                return None
    return None


def cpu_baseline(fields, max_seconds=25.0, warmup=1, steps=2):
    """Time the CPU path on a bounded sample; returns (fields/s, kind, cores, sample-note)."""
    from oracle import polybin_oracle as O
    nthreads = os.cpu_count()
    ref_utils = load_ref_utils()
    base = O.OracleBase([L] * 3, [N] * 3, pixel_window="tsc", nthreads=nthreads)
    bs = O.OracleBSpec(base, EDGES, lmax=LMAX)
    # probe: the per-field part (FFTs, filters) and the cost of 2% of the triplets
    t = time.perf_counter()
    cpu_reference_step(bs, 0.0, fields[0], nthreads, ref_utils)
    t_field = time.perf_counter() - t
    t = time.perf_counter()
    cpu_reference_step(bs, 0.02, fields[0], nthreads, ref_utils)
    t_trip = max(1e-6, time.perf_counter() - t - t_field) / 0.02
    budget = max_seconds / (warmup + steps)
    frac = 1.0
    for f in (1.0, 0.5, 0.25, 0.125, 0.0625, 0.03125):
        frac = f
        if t_field + f * t_trip <= budget:
            break
    for i in range(warmup):
        cpu_reference_step(bs, frac, fields[i % len(fields)], nthreads, ref_utils)
    ts = []
    for i in range(steps):
        t = time.perf_counter()
        cpu_reference_step(bs, frac, fields[i % len(fields)], nthreads, ref_utils)
        ts.append(time.perf_counter() - t)
    ts = float(np.median(ts))
    # a field = the FFT/filter part once + all triplets; only the triplet sum is sampled
    per_field = ts + (1.0 - frac) * t_trip
    kind = "reference" if ref_utils is not None else "port"
    note = ("one 256^3 field per step: 32 FP64 c2r (scipy) + %s over %.1f%% of the 888 triplets; "
            "fields/s = 1 / (step time + unsampled triplets at the probed rate), median of %d after %d warm-up"
            % ("reference assemble_b3 (oracle/_ref)" if ref_utils else "oracle C triplet loop",
               100 * frac, steps, warmup))
    return 1.0 / per_field, kind, nthreads, note


def run_reference(args, rank, world):
    if rank != 0:
        return
    from polybin3d_b200 import synthetic
    fields = [synthetic.lognormal(N, L, seed=s) for s in range(2)]
    v, kind, cores, note = cpu_baseline(fields, max_seconds=max(30.0, 4.0 * (args.steps + args.warmup)),
                                        warmup=args.warmup, steps=args.steps)
    line = {"metric": METRIC, "value": v, "unit": "fields/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded float32 lognormal fields)",
            "config": {"workload": WORKLOAD}, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "fields/s", "cores": cores, "kind": kind, "sample": note},
            "e2e": {"value": v, "unit": "fields/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if args.workload == "headline":
        # the metric's second half on the host: one Monte Carlo Fisher realisation per workload
        line["fisher"] = {name: fisher_reference_line(name) for name in ("fisher_pk128", "fisher_bk128")}
    print(json.dumps(line))


def run_ours(args, rank, world, local):
    import contextlib
    import io

    import torch
    import polybin3d_b200 as pb
    from polybin3d_b200 import _native as nat
    from polybin3d_b200 import autotune
    from polybin3d_b200 import synthetic

    dev = torch.device("cuda", local)
    with contextlib.redirect_stdout(io.StringIO()):
        base = pb.PolyBin3D([L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
        bs = pb.BSpec(base, EDGES, lmax=LMAX, contraction=args.contraction)
        bs.compute_fisher_ideal()  # one-off, cached (as the reference caches it)
    method = bs._method(torch.float32)
    inv_fish = torch.as_tensor(bs.inv_fish_ideal, device=dev)
    norm = torch.as_tensor(base.volume / float(N ** 3) / bs.sym_factor, device=dev)

    n_pool = 4
    host = [torch.from_numpy(synthetic.lognormal(N, L, seed=1000 * rank + s)).pin_memory() for s in range(n_pool)]
    resident = [h.to(dev) for h in host]
    torch.cuda.synchronize()

    # device-resident step: the Bk_ideal numerator + F^-1, no host sync
    cev = []
    used = {}

    route = {}

    def step(i, record=False):
        # the public Bk_ideal path (BSpec._b3_sums): with the tensor-core contraction, the route
        # (g-maps into a tiled set, or plain maps) the autotuner found faster for this shape
        x = resident[i % n_pool]
        f32 = torch.float32
        xk = bs._data_spectrum(x, keep64=True)  # FP64 transform, read as it is by the synthesis
        w = bs._data_weight(f32)
        idx = bs._triplet_index()
        if "tiled" not in route:
            ok = bs._tiled_ok(f32)
            route["tiled"] = ok and (bs._b3_route(xk, w, 1.0, f32) == "tiled" if args.route == "auto"
                                     else args.route == "tiled")
        tiled = route["tiled"]
        if tiled:
            G = bs._g_maps_tiled(xk, w, 1.0, f32)
            plan = bs._plan("b3", G.n_maps, G.n_maps, G.n_maps, idx)
            run = lambda: autotune.contract_tiled(plan, G, out, base.ws, bs._grid_scale(G.shape))
        else:
            G = bs._g_maps(xk, w, 1.0, rd=f32)
            plan = bs._plan("b3", G.shape[0], G.shape[0], G.shape[0], idx)
            run = lambda: autotune.contract(plan, G, G, G, out, base.ws, method, 1.0)
        used["plan"] = plan
        out = torch.empty(plan.n_trip, dtype=torch.float64, device=dev)
        if record:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        run()
        if record:
            e1.record()
            cev.append((e0, e1))
        return inv_fish @ (out * norm)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = nat.LAUNCHES[0]
    with Clocks(local) as clk:
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for i in range(args.steps):
            res = step(i, record=True)
        t1.record()
        torch.cuda.synchronize()
    launches = nat.LAUNCHES[0] - l0  # kernels of libpb_b200 (cuFFT and torch launches not counted)
    ms = t0.elapsed_time(t1)
    kern_ms = float(np.mean([a.elapsed_time(b) for a, b in cev]))
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * args.steps / (ms / 1000.0)

    # end-to-end through the public API from pinned host memory: Bk_ideal on the list of
    # the step's fields (each field's H2D copy and result read-back inside the timed region;
    # copies overlap the previous field's estimator)
    with contextlib.redirect_stdout(io.StringIO()):
        bs.Bk_ideal([host[i % n_pool] for i in range(args.warmup)])
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    with contextlib.redirect_stdout(io.StringIO()):
        r = bs.Bk_ideal([host[i % n_pool] for i in range(args.steps)])
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        tt = torch.tensor([e2e_ms], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    e2e = world * args.steps / (e2e_ms / 1000.0)

    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        bf16 = float(peaks.get("bf16_tflops", 1590.0))
        n_vox = int(np.prod(bs.map_grid))
        # every map read once: 4 bytes per voxel (FP32) for plain maps; a tiled set is
        # [FP32 pair factors][bf16 hi + lo C operand] per 128-voxel tile
        tiled = route.get("tiled", False)
        alg_bytes = (nat.tiled_maps_bytes(bs.Nl * bs.Nk_squeeze, bs.Nk_squeeze, n_vox) if tiled
                     else bs.Nl * bs.Nk_squeeze * n_vox * 4)
        plan = used["plan"]
        # GEMM form D[c, pair] = sum_x C_c(x) (A B)_pair(x) on the map grid, and the useful
        # triple products (3 flops per voxel and triplet)
        gemm_flops = 2.0 * plan.n_c * plan.n_pairs * n_vox
        useful_flops = 3.0 * n_vox * plan.n_trip
        achieved = gemm_flops / (kern_ms / 1000.0) / 1e12
        achieved_hbm = alg_bytes / (kern_ms / 1000.0) / 1e9
        line = {"metric": METRIC, "value": value, "unit": "fields/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 maps / fp64 sums",
                "data": "synthetic (seeded float32 lognormal fields, pool of 4 per rank)",
                "config": {"workload": WORKLOAD, "contraction": ("tc, tiled set" if tiled else "tc") if method == nat.PB_TRIPLET_TC else "simt",
                           "map_grid": list(bs.map_grid),
                           "l2": "inputs+intermediates 4.4 GB/step >> 126 MB L2", "parallelism": "replicas"},
                "e2e": {"value": e2e, "unit": "fields/s", "h2d_bytes_per_step": N ** 3 * 4,
                        "d2h_bytes_per_step": bs.N_bins * 8},
                "gpu_launches": launches,
                # the contraction reads every map once and does 68 GEMM flops per byte, below
                # the ridge of the measured peaks (~250 flop/B): HBM is its binding roofline;
                # the tensor-core (GEMM-form) figures are kept beside it
                "roofline": {"bound": "hbm", "kernel": "triplet contraction (tcgen05)", "achieved": achieved_hbm,
                             "peak": hbm, "unit": "GB/s", "frac": achieved_hbm / hbm,
                             "traffic": (TC_TRAFFIC_TILED if tiled else TC_TRAFFIC_PLAIN) if method == nat.PB_TRIPLET_TC else None,
                             "alg_bytes_per_launch": alg_bytes, "kernel_ms": kern_ms,
                             "gemm_flops_per_launch": gemm_flops, "gemm_tflops": achieved,
                             "gemm_peak_tflops": bf16, "frac_tensor": achieved / bf16,
                             "useful_flops_per_launch": useful_flops,
                             "useful_tflops": useful_flops / (kern_ms / 1000.0) / 1e12,
                             "peak_source": ("of measured: MEASURED_PEAKS.json hbm_gbs and bf16_tflops (burst)"
                                             if peaks else "of fallback: 6650 GB/s and 1590 TFLOP/s")},
                "clocks": clk.summary()}
        if not args.no_cpu_baseline and world == 1:
            v, kind, cores, note = cpu_baseline([host[0].numpy(), host[1].numpy()])
            line["cpu_baseline"] = {"value": v, "unit": "fields/s", "cores": cores, "kind": kind, "sample": note}
    # the metric's second half: Monte Carlo Fisher realisations/s at 128^3 (Pk and Bk), every
    # rank taking part (the seeds are shared over the ranks)
    del bs, base, resident
    torch.cuda.empty_cache()
    if args.workload == "headline":
        fisher = {}
        for name in ("fisher_pk128", "fisher_bk128"):
            fisher[name] = fisher_measure(name, FISHER_STEPS, 3, rank, world, local, not args.no_cpu_baseline)
        if rank == 0:
            line["fisher"] = fisher
    if rank == 0:
        print(json.dumps(line))


def fisher_alg_bytes(kind, N, n_bins):
    """Compulsory HBM bytes of one FP64 Monte Carlo realisation, each kernel reading its
    inputs and writing its outputs once and each 3D FFT counted as one read + one write
    (N^3 voxels of 8 B, N^3/2 half modes of 16 B).
    Pk, per Fisher row: Q spectrum write (8 N^3), c2r (8 + 8), mask product (24), r2c (8 + 8),
    CROSS reduction read (8): 72 N^3.
    Bk, per bin: three accumulating leg passes (3 x 16 N^3), the S^-1 P mask filter of its
    Q (c2r 16, mask 24, r2c 16) and its rows' read (8): 112 N^3."""
    per = 72 if kind == "pk" else 112
    return float(per) * N ** 3 * n_bins


def fisher_cpu_baseline(cfg, kind):
    """The oracle port of the reference's Monte Carlo Fisher contribution (FP64, scipy FFTs
    with all host threads) for one realisation on the reference's MT19937 noise."""
    from oracle import polybin_oracle as O
    nthreads = os.cpu_count()
    N, L = cfg["N"], cfg["L"]
    ref_utils = load_ref_utils()
    ob = O.OracleBase([L] * 3, [N] * 3, nthreads=nthreads, kernels=ref_utils)
    m = fisher_mask(N, L).astype(np.float64)
    if kind == "pk":
        est = O.OraclePSpec(ob, cfg["edges"], lmax=cfg["lmax"], mask=m)
        est.fisher_contribution(ob.reference_noise(int(1e7)))  # warm-up
        ts = []
        for s in (1, 2):
            t = time.perf_counter()
            est.fisher_contribution(ob.reference_noise(s + int(1e7)))
            ts.append(time.perf_counter() - t)
        note = ("seeds 1, 2 after one warm-up, median, (the reference's MT19937 noise) through the "
                "compute_fisher_contribution flow restated in the oracle")
        return 1.0 / float(np.median(ts)), "reference" if ref_utils is not None else "port", nthreads, (
            note + (", with the reference's compiled filter / integration kernels (oracle/_ref)" if ref_utils
                    is not None else ", numpy kernels") + ", scipy FFT workers=%d" % nthreads)
    else:
        est = O.OracleBSpec(ob, cfg["edges"], lmax=cfg["lmax"], mask=m)
        sym = est.symmetry_factor()  # cached once, as the reference caches it
        t = time.perf_counter()
        est.fisher_contribution(ob.reference_noise(int(1e7)), ob.reference_noise(int(2e7)), sym=sym)
    dt = time.perf_counter() - t
    note = ("one realisation (seed 0, the reference's MT19937 noise): the compute_fisher_contribution flow "
            "restated in the oracle, %s, scipy FFT workers=%d; single timing"
            % ("with the reference's compiled filter / integration kernels (oracle/_ref)" if ref_utils is not None
               else "numpy kernels", nthreads))
    return 1.0 / dt, "reference" if ref_utils is not None else "port", nthreads, note


def fisher_reference_line(name):
    """The reference arm of one Monte Carlo Fisher workload (rank 0; host cores only)."""
    cfg = FISHER[name]
    kind = "pk" if name.startswith("fisher_pk") else "bk"
    v, k, cores, note = fisher_cpu_baseline(cfg, kind)
    return {"metric": cfg["metric"], "value": v, "unit": "sims/s", "ms_per_step": 1000.0 / v,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic (Gaussian random fields, shell-sector mask)",
            "config": {"workload": cfg["workload"]}, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "sims/s", "cores": cores, "kind": k, "sample": note},
            "e2e": {"value": v, "unit": "sims/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def fisher_measure(name, steps, warmup, rank, world, local, with_cpu):
    """Monte Carlo Fisher throughput of one workload: `value` = realisations/s with the
    white noise drawn on the device (one captured CUDA graph per batch), `e2e` = the
    reference-identical path (the reference's MT19937 noise drawn by host workers, copied
    in, the Fisher matrix read back).  Timed with CUDA events on the current stream, max
    over ranks; seeds are shared round-robin over the ranks."""
    import contextlib
    import io

    import torch
    import polybin3d_b200 as pb
    from polybin3d_b200 import _native as nat

    cfg = FISHER[name]
    kind = "pk" if name.startswith("fisher_pk") else "bk"
    dev = torch.device("cuda", local)
    N, L, B = cfg["N"], cfg["L"], cfg["batch"]
    with contextlib.redirect_stdout(io.StringIO()):
        base = pb.PolyBin3D([L] * 3, [N] * 3, backend="cuda")
        m = fisher_mask(N, L)
        if kind == "pk":
            est = pb.PSpec(base, cfg["edges"], lmax=cfg["lmax"], mask=m)
        else:
            est = pb.BSpec(base, cfg["edges"], lmax=cfg["lmax"], mask=m)

    def fisher(n_it, noise):
        with contextlib.redirect_stdout(io.StringIO()):
            if kind == "pk":
                return est.compute_fisher(n_it, batch=B, noise=noise)
            return est.compute_fisher(n_it, noise=noise)

    def max_over_ranks(x):
        if world > 1:
            tt = torch.tensor([x], device=dev)
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            return float(tt.item())
        return x

    per_step = B * world  # realisations per step over all ranks
    fisher(max(3, warmup) * per_step, "philox")  # capture + warm-up replays
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = nat.LAUNCHES[0]
    with Clocks(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fisher(steps * per_step, "philox")
        e1.record()
        torch.cuda.synchronize()
    launches = nat.LAUNCHES[0] - l0
    ms = max_over_ranks(e0.elapsed_time(e1))
    value = steps * per_step / (ms / 1000.0)

    # end to end: the reference-identical path (the reference's MT19937 draws made on host
    # worker processes, copied in; the Fisher matrix read back)
    n_e2e = max(2, steps) * per_step
    fisher(per_step * 4, "reference")  # worker start-up and warm-up
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0.record()
    fisher(n_e2e, "reference")
    e1.record()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
    e2e = n_e2e / e2e_s
    rec = None
    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        alg = fisher_alg_bytes(kind, N, est.N_bins)
        achieved = alg / (ms / 1000.0 / (steps * B)) / 1e9
        fields = 1 if kind == "pk" else 2
        rec = {"metric": cfg["metric"], "value": value, "unit": "sims/s", "n_gpus": world, "steps": steps,
               "warmup": warmup, "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64",
               "data": "synthetic (Gaussian random fields drawn on the device, shell-sector mask)",
               "config": {"workload": cfg["workload"], "n_bins": est.N_bins, "realisations_per_step": per_step,
                          "graph": "one captured CUDA graph per batch of %d" % B,
                          "l2": "per-realisation working set > 3 GB >> 126 MB L2",
                          "parallelism": "seeds round-robin over ranks" if world > 1 else "single GPU"},
               "e2e": {"value": e2e, "unit": "sims/s",
                       "h2d_bytes_per_step": per_step * fields * 2 * N ** 3 * 8,
                       "d2h_bytes_per_step": est.N_bins ** 2 * 8,
                       "path": "compute_fisher(noise='reference'): the reference's MT19937 draws on host workers"},
               "gpu_launches": launches,
               "roofline": {"bound": "hbm", "kernel": "whole realisation (FFTs, filters, reductions)",
                            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                            "traffic": None, "alg_bytes_per_realisation": alg,
                            "peak_source": "of measured: MEASURED_PEAKS.json hbm_gbs" if peaks else "of fallback: 6650"},
               "clocks": clk.summary()}
        if with_cpu and world == 1:
            v, k, cores, note = fisher_cpu_baseline(cfg, kind)
            rec["cpu_baseline"] = {"value": v, "unit": "sims/s", "cores": cores, "kind": k, "sample": note}
    del est, base
    torch.cuda.empty_cache()
    return rec


def run_fisher(args, rank, world, local):
    if args.impl == "reference":
        if rank == 0:
            line = fisher_reference_line(args.workload)
            line.update({"n_gpus": args.gpus, "steps": 1, "warmup": 0, "scaling": "weak", "vs_baseline": None})
            print(json.dumps(line))
        return
    rec = fisher_measure(args.workload, args.steps, args.warmup, rank, world, local, not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(rec))


def run_bk512(args, rank, world, local):
    """Forward + gradient at 512^3: per field, Bk = F_ideal^-1 num(d) and the VJP J^T v
    (v a fixed random cotangent) through polybin3d_b200.autograd.BkNumerator."""
    import contextlib
    import io

    import torch
    import polybin3d_b200 as pb
    from polybin3d_b200 import _native as nat
    from polybin3d_b200 import synthetic
    from polybin3d_b200.autograd import bk_numerator

    cfg = BK512
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no gradient path; its 512^3 "
                              "numerator needs 48 FP64 maps (48 GB of host memory) per field"}))
        return
    dev = torch.device("cuda", local)
    N, L = cfg["N"], cfg["L"]
    with contextlib.redirect_stdout(io.StringIO()):
        base = pb.PolyBin3D([L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
        bs = pb.BSpec(base, cfg["edges"], lmax=cfg["lmax"], contraction=args.contraction)
        t0 = time.perf_counter()
        bs.compute_fisher_ideal()  # one-off, cached (as the reference caches it)
        t_fisher = time.perf_counter() - t0
    inv_fish = torch.as_tensor(bs.inv_fish_ideal, device=dev)
    n_pool = 2
    host = [torch.from_numpy(synthetic.lognormal(N, L, seed=1000 * rank + s)).pin_memory() for s in range(n_pool)]
    resident = [h.to(dev) for h in host]
    v = torch.as_tensor(np.random.default_rng(0).standard_normal(bs.N_bins), device=dev)

    def step(x):
        x = x.detach().requires_grad_(True)
        bk = inv_fish @ bk_numerator(bs, x)
        (g,) = torch.autograd.grad(bk, x, grad_outputs=v)
        return bk.detach(), g

    for i in range(args.warmup):
        step(resident[i % n_pool])
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = nat.LAUNCHES[0]
    with Clocks(local) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(args.steps):
            step(resident[i % n_pool])
        e1.record()
        torch.cuda.synchronize()
    launches = nat.LAUNCHES[0] - l0
    ms = e0.elapsed_time(e1)
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * args.steps / (ms / 1000.0)
    # end to end: pinned host field in, Bk and the gradient map back to pinned host memory
    g_host = torch.empty((N, N, N), dtype=torch.float32).pin_memory()
    bk_host = torch.empty(bs.N_bins, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()
    e0.record()
    for i in range(args.steps):
        x = host[i % n_pool].to(dev, non_blocking=True)
        bk, g = step(x)
        bk_host.copy_(bk, non_blocking=True)
        g_host.copy_(g, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        tt = torch.tensor([e2e_ms], device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    if rank == 0:
        print(json.dumps({"metric": cfg["metric"], "value": value, "unit": "fields/s", "n_gpus": world,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f32 maps / fp64 sums", "data": "synthetic (seeded float32 lognormal fields)",
                          "config": {"workload": cfg["workload"], "n_bins": bs.N_bins, "maps": bs.Nl * bs.Nk_squeeze,
                                     "map_grid": list(bs.map_grid), "ideal_fisher_setup_s": t_fisher,
                                     "l2": "inputs+intermediates > 40 GB/step >> 126 MB L2",
                                     "parallelism": "replicas" if world > 1 else "single GPU"},
                          "e2e": {"value": world * args.steps / (e2e_ms / 1000.0), "unit": "fields/s",
                                  "h2d_bytes_per_step": N ** 3 * 4, "d2h_bytes_per_step": N ** 3 * 4 + bs.N_bins * 8},
                          "gpu_launches": launches, "clocks": clk.summary()}))


def main():
    args = parse()
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        # host cores only: rank 0 runs the reference's CPU path, the other ranks exit
        if args.workload == "bk512grad":
            run_bk512(args, rank, world, local)
        elif args.workload not in ("headline", "bk256"):
            run_fisher(args, rank, world, local)
        else:
            run_reference(args, rank, world)
        return
    import datetime

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    try:
        if args.workload == "bk512grad":
            run_bk512(args, rank, world, local)
        elif args.workload not in ("headline", "bk256"):
            run_fisher(args, rank, world, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
