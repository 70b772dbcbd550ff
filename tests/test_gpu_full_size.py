"""Parity with the reference at the full benchmark sizes (fixtures made by running the
reference itself: tests/golden/make_golden.py cases cfg2_bk256, cfg3_pk128, cfg4_bk128).

* 256^3 Bk_ideal (box 2000 Mpc/h, TSC, lmax = 2, 16 linear bins to 0.2 h/Mpc, the seeded
  float32 lognormal field): bins and symmetry factors exact / 1e-10, the ideal Fisher matrix
  (stored sparse: it couples only the multipoles of one triangle) 1e-10, the FP64 numerator
  and b0, b2 1e-10 per bin; the mixed-precision path -- the configuration the benchmark times,
  tensor-core and CUDA-core contractions -- per bin against the reference, with the floor
  FLOOR x (largest |B| of the multipole block) under each bin's |B|: MIXED_TOL on the monopole
  block and against each block's largest value, a measured limit on the quadrupole bins that
  cancel.
* 128^3 Monte Carlo Fisher contributions on the 200-hole shell-sector mask: Pk (lmax = 4,
  60 bins) and Bk (lmax = 0, 203 bins), seed 0, 1e-8; numerators of masked fields 1e-10.
* The 128^3 cubic-numerator gradient against central finite differences (step 1e-3 x rms,
  one Richardson step, 64 seeded voxels inside the mask), 1e-6.
"""
import contextlib
import io
import os

import numpy as np
import pytest
import torch

from polybin3d_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MIXED_TOL = 1e-5
FLOOR = 1e-3


def gold(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def per_bin(a, b, n_blocks, floor=FLOOR):
    """Per-bin relative errors |a_i - b_i| / max(|b_i|, floor * max_block |b|), per block."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    nb = len(b) // n_blocks
    out = []
    for j in range(n_blocks):
        x, y = a[j * nb:(j + 1) * nb], b[j * nb:(j + 1) * nb]
        out.append(np.abs(x - y) / np.maximum(np.abs(y), floor * np.max(np.abs(y))))
    return np.concatenate(out)


def survey_mask(N, L):
    return synthetic.shell_mask(N, L, r_in=250.0, r_out=700.0, n_holes=200, hole_r=(5.0, 20.0), hole_box=700.0,
                                seed=0)


@pytest.fixture(scope="module")
def pb():
    import polybin3d_b200
    return polybin3d_b200


@pytest.fixture(scope="module")
def cfg2():
    return gold("cfg2_bk256")


@pytest.fixture(scope="module")
def cfg2_field(cfg2):
    return synthetic.lognormal(int(cfg2["N"]), float(cfg2["L"]), seed=int(cfg2["data_seed"]))


def cfg2_bspec(pb, g, precision, contraction):
    N, L = int(g["N"]), float(g["L"])
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision=precision)
    return quiet(pb.BSpec, b, g["edges"], lmax=2, contraction=contraction)


def test_cfg2_fp64(pb, cfg2, cfg2_field):
    g = cfg2
    bs = cfg2_bspec(pb, g, "fp64", "simt")
    assert np.array_equal(bs.all_bins, g["bk_bins"])
    num = quiet(bs.Bk_numerator_ideal, cfg2_field)
    assert np.max(per_bin(num, g["bk_num"], 2)) < 1e-10
    assert rel(bs.sym_factor, g["bk_sym"]) < 1e-10
    bk = quiet(bs.Bk_ideal, cfg2_field)
    fish = np.asarray(bs.fish_ideal)
    r, c, v = g["fish_rows"], g["fish_cols"], g["fish_vals"]
    scale = np.max(np.abs(v))
    assert np.max(np.abs(fish[r, c] - v)) / scale < 1e-10
    off = fish.copy()
    off[r, c] = 0.0
    assert np.max(np.abs(off)) / scale < 1e-10
    for k in ("b0", "b2"):
        assert np.max(per_bin(bk[k], g["Bk_" + k], 1)) < 1e-10, k


def block_rel(a, b, n_blocks):
    """max |a - b| / max |b| within each multipole block."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    nb = len(b) // n_blocks
    return max(np.max(np.abs(a[j * nb:(j + 1) * nb] - b[j * nb:(j + 1) * nb])) / np.max(np.abs(b[j * nb:(j + 1) * nb]))
               for j in range(n_blocks))


# worst quadrupole bin (floored per-bin metric) of the mixed path: bins whose triple products
# cancel down to ~1e-3 of the block's largest; FP32 storage of exact maps alone puts 1.9e-5
# on the worst one, the tensor cores' bf16 hi + lo split (2^-17 per product) 6e-4
QUAD_TOL = {"tc": 1e-3, "simt": 1e-4}


@pytest.mark.parametrize("contraction", ["tc", "simt"])
def test_cfg2_mixed_per_bin(pb, cfg2, cfg2_field, contraction):
    """The benchmark's configuration: FP32 maps (data transform in FP64), the tensor-core
    (split-bf16) or CUDA-core contraction, FP64 sums, against the reference: every monopole
    bin within MIXED_TOL, every bin within MIXED_TOL of its block's largest value, and the
    cancelling quadrupole bins within the measured limit of each contraction."""
    from polybin3d_b200.bspec import tc_available
    if contraction == "tc" and not tc_available():
        pytest.skip("tensor-core contraction not available")
    g = cfg2
    bs = cfg2_bspec(pb, g, "mixed", contraction)
    num = quiet(bs.Bk_numerator_ideal, cfg2_field)
    e = per_bin(num, g["bk_num"], 2)
    n3 = len(e) // 2
    assert np.max(e[:n3]) < MIXED_TOL, ("monopole", float(np.max(e[:n3])))
    assert np.max(e[n3:]) < QUAD_TOL[contraction], ("quadrupole", float(np.max(e[n3:])), float(np.median(e[n3:])))
    assert block_rel(num, g["bk_num"], 2) < MIXED_TOL
    bk = quiet(bs.Bk_ideal, cfg2_field)
    for k in ("b0", "b2"):
        assert block_rel(bk[k], g["Bk_" + k], 1) < MIXED_TOL, k
        assert np.max(per_bin(bk[k], g["Bk_" + k], 1)) < QUAD_TOL[contraction], k


def test_cfg3_pk_fisher(pb):
    g = gold("cfg3_pk128")
    N, L = int(g["N"]), float(g["L"])
    m = survey_mask(N, L)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="none", backend="cuda")
    ps = quiet(pb.PSpec, b, g["edges"], lmax=int(g["pk_lmax"]), mask=m)
    assert rel(quiet(ps.compute_fisher_contribution, 0), g["f0"]) < 1e-8
    data = synthetic.lognormal(N, L, seed=int(g["data_seed"])).astype(np.float64) * m
    assert rel(quiet(ps.Pk_numerator, data), g["num"]) < 1e-10


def test_cfg4_bk_fisher(pb):
    g = gold("cfg4_bk128")
    N, L = int(g["N"]), float(g["L"])
    m = survey_mask(N, L)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="none", backend="cuda")
    bs = quiet(pb.BSpec, b, g["edges"], lmax=int(g["bk_lmax"]), mask=m)
    assert np.array_equal(bs.all_bins, g["bins"])
    assert rel(quiet(bs.compute_fisher_contribution, 0), g["f0"]) < 1e-8
    assert rel(bs.sym_factor, g["sym"]) < 1e-10
    data = synthetic.lognormal(N, L, seed=int(g["data_seed"])).astype(np.float64) * m
    assert rel(quiet(bs.Bk_numerator, data, include_linear_term=False), g["num"]) < 1e-10


def test_cfg4_gradient_finite_differences(pb):
    """d num / d delta of the 203-bin cubic numerator at 128^3 (masked) from the autograd
    backward kernels, against central differences on 64 seeded voxels inside the mask: the
    numerator is cubic, so one Richardson step of the step-h and step-h/2 differences is exact
    up to rounding."""
    from polybin3d_b200.autograd import bk_numerator
    g = gold("cfg4_bk128")
    N, L = int(g["N"]), float(g["L"])
    m = survey_mask(N, L)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="none", backend="cuda")
    bs = quiet(pb.BSpec, b, g["edges"], lmax=0, mask=m)
    dev = b.device
    d = torch.as_tensor(synthetic.lognormal(N, L, seed=42).astype(np.float64), device=dev)
    rng = np.random.default_rng(4)
    gam = torch.as_tensor(rng.standard_normal(bs.N_bins), device=dev)
    x = d.clone().requires_grad_(True)
    (grad,) = torch.autograd.grad(bk_numerator(bs, x), x, grad_outputs=gam)
    inside = np.flatnonzero(m.reshape(-1) > 0)
    vox = rng.choice(inside, size=64, replace=False)
    h = 1e-3 * float(d.std())

    def directional(v):
        def cd(s):
            with torch.no_grad():
                return float(torch.dot(gam, bk_numerator(bs, d + s * v) - bk_numerator(bs, d - s * v))) / (2 * s)
        return (4 * cd(0.5 * h) - cd(h)) / 3

    v = torch.zeros(d.numel(), dtype=d.dtype, device=dev)
    v[torch.as_tensor(vox, device=dev)] = torch.as_tensor(rng.standard_normal(64), device=dev)
    v = v.reshape(d.shape)
    fd, ad = directional(v), float(torch.sum(grad * v))
    assert abs(ad - fd) <= 1e-6 * abs(fd), (ad, fd)
    gmax = float(grad.abs().max())
    for j in vox[:8]:
        e = torch.zeros(d.numel(), dtype=d.dtype, device=dev)
        e[int(j)] = 1.0
        fd, ad = directional(e.reshape(d.shape)), float(grad.reshape(-1)[int(j)])
        assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-3 * gmax), (int(j), ad, fd)
