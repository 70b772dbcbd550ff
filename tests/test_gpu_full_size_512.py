"""The 512^3 workload (box 4000 Mpc/h, TSC, lmax = 2, 24 linear bins to 0.35 h/Mpc: 2756
triangle bins from 48 maps on the full 512^3 grid), checked where no reference run fits:

* the mixed-precision forward the 512^3 benchmark streams (FP32 transforms and maps,
  tensor-core contraction, FP64 sums) against the FP64 path on one lognormal field, per bin
  with the floor 1e-3 x (largest |B| of the multipole block): monopole bins within MIXED_TOL,
  quadrupole bins (some cancel) within QUAD_TOL, every bin within MIXED_TOL of its block's
  largest value;
* the FP64 triplet sums of the device against the reference's own compiled assemble_b3
  (utils.pyx:614-636, built into oracle/_ref) on the same FP64 maps, for the triplets of a
  sample of bins (the reference holds all 48 maps of a field in host memory: 51 GB);
* the FP64 gradient (bin-filtered maps recomputed in the backward) against central finite
  differences on 64 seeded voxels (one Richardson step: exact for a cubic), 1e-6, and the
  mixed-precision gradient against it.
Needs about 120 GB of device memory."""
import contextlib
import importlib.util
import io
import os

import numpy as np
import pytest
import torch

from polybin3d_b200 import synthetic

pytestmark = pytest.mark.gpu
N, L = 512, 4000.0
EDGES = np.linspace(2 * np.pi / L, 0.35, 25)
MIXED_TOL = 1e-5
QUAD_TOL = 1e-3  # quadrupole bins whose triple products cancel (the split-bf16 contraction's limit)
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def per_bin(a, b, n_blocks, floor=1e-3):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    nb = len(b) // n_blocks
    return np.concatenate([np.abs(a[j * nb:(j + 1) * nb] - b[j * nb:(j + 1) * nb]) /
                           np.maximum(np.abs(b[j * nb:(j + 1) * nb]), floor * np.max(np.abs(b[j * nb:(j + 1) * nb])))
                           for j in range(n_blocks)])


def free():
    import gc
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


@pytest.fixture(scope="module")
def field():
    return synthetic.lognormal(N, L, seed=0)


@pytest.fixture(scope="module")
def fp64_result(field):
    """FP64 numerator and the FP64 sums of a sample of triplets with the maps they use."""
    import polybin3d_b200 as pb
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="fp64")
    bs = quiet(pb.BSpec, b, EDGES, lmax=2, contraction="simt")
    assert bs.N_bins == 2756 and tuple(bs.map_grid) == (N, N, N)
    bs.sym_factor = np.ones(bs.N_bins)  # raw sums: the symmetry factors are checked at 256^3
    num = quiet(bs.Bk_numerator_ideal, field)
    S = [0, 5, 11, 17, 23]
    ab = bs.all_bins
    sel = np.flatnonzero(np.isin(ab[:, 0], S) & np.isin(ab[:, 1], S) & np.isin(ab[:, 2], S))
    x = b.as_device(field.astype(np.float64))
    xk = b.to_fourier(x)
    G = bs._g_maps(xk, bs._data_weight(torch.float64), 1.0 / bs.cube_mask_mean ** (1. / 3.))
    sums = bs._contract('b3', G, G, G, bs._triplet_index()).cpu().numpy()[sel]
    g_host = np.empty((bs.Nl, len(S)) + (N, N, N), dtype=np.float64)
    for l in range(bs.Nl):
        for j, k in enumerate(S):
            g_host[l, j] = G[l * bs.Nk_squeeze + k].cpu().numpy()
    sub = ab[sel].copy()
    remap = {k: j for j, k in enumerate(S)}
    for c in range(3):
        sub[:, c] = [remap[int(v)] for v in sub[:, c]]
    del G, x, xk, bs, b
    free()
    return num, sums, g_host, np.ascontiguousarray(sub)


def test_512_mixed_forward_per_bin(field, fp64_result):
    import polybin3d_b200 as pb
    from polybin3d_b200.bspec import tc_available
    ref = fp64_result[0]
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
    bs = quiet(pb.BSpec, b, EDGES, lmax=2, contraction="tc" if tc_available() else "simt")
    bs.sym_factor = np.ones(bs.N_bins)
    num = quiet(bs.Bk_numerator_ideal, field)
    del bs, b
    free()
    e = per_bin(num, ref, 2)
    n3 = len(ref) // 2
    assert np.max(e[:n3]) < MIXED_TOL, ("monopole", float(np.max(e[:n3])), float(np.median(e[:n3])))
    assert np.max(e[n3:]) < QUAD_TOL, ("quadrupole", float(np.max(e[n3:])), float(np.median(e[n3:])))
    for j in range(2):
        blk = slice(j * n3, (j + 1) * n3)
        assert np.max(np.abs(num[blk] - ref[blk])) / np.max(np.abs(ref[blk])) < MIXED_TOL, j


def test_512_fp64_sums_match_reference_assemble_b3(fp64_result):
    d = os.path.join(REPO, "oracle", "_ref")
    so = [f for f in os.listdir(d) if f.startswith("pb_ref_utils") and f.endswith(".so")] if os.path.isdir(d) else []
    if not so:
        pytest.skip("the reference's compiled kernels (oracle/_ref) are not built")
    spec = importlib.util.spec_from_file_location("pb_ref_utils", os.path.join(d, so[0]))
    ref_utils = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref_utils)
    _, sums, g_host, sub = fp64_result
    assert len(sub) >= 10
    ref = ref_utils.assemble_b3(g_host, sub, os.cpu_count())
    assert np.max(np.abs(sums - ref)) / np.max(np.abs(ref)) < 1e-10


def test_512_gradient(field):
    """FP64 vector-Jacobian product against Richardson finite differences on 64 voxels, and
    the mixed-precision product (FP32 maps, the benchmark's gradient) against the FP64 one."""
    import polybin3d_b200 as pb
    from polybin3d_b200.autograd import bk_numerator
    rng = np.random.default_rng(7)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="fp64")
    bs = quiet(pb.BSpec, b, EDGES, lmax=2, contraction="simt")
    bs.sym_factor = np.ones(bs.N_bins)
    dev = b.device
    d = torch.as_tensor(field.astype(np.float64), device=dev)
    gam = torch.as_tensor(rng.standard_normal(bs.N_bins), device=dev)
    x = d.clone().requires_grad_(True)
    (g64,) = torch.autograd.grad(bk_numerator(bs, x), x, grad_outputs=gam)
    del x
    vox = rng.choice(d.numel(), size=64, replace=False)
    v = torch.zeros(d.numel(), dtype=torch.float64, device=dev)
    v[torch.as_tensor(vox, device=dev)] = torch.as_tensor(rng.standard_normal(64), device=dev)
    v = v.reshape(d.shape)
    h = 1e-3 * float(d.std())

    def cd(s):
        with torch.no_grad():
            return float(torch.dot(gam, bk_numerator(bs, d + s * v) - bk_numerator(bs, d - s * v))) / (2 * s)
    fd = (4 * cd(0.5 * h) - cd(h)) / 3
    ad = float(torch.sum(g64 * v))
    assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)
    g64_host = g64.cpu()
    del g64, bs, b, d, v
    free()
    bm = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
    bsm = quiet(pb.BSpec, bm, EDGES, lmax=2)
    bsm.sym_factor = np.ones(bsm.N_bins)
    xm = torch.as_tensor(field, device=bm.device).requires_grad_(True)
    (gm,) = torch.autograd.grad(bk_numerator(bsm, xm), xm, grad_outputs=gam.to(bm.device))
    gm = gm.double().cpu()
    scale = float(g64_host.abs().max())
    assert float((gm - g64_host).abs().max()) / scale < 1e-4
