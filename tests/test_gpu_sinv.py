"""A caller's S^-1 weighting (PSpec(applySinv=..., applySinv_transpose=...)) through the CUDA
path, against the reference run with the same filter (tests/golden/custom_sinv.npz): the
non-symmetric S^-1 = IFT w(k) FT u of tests/golden/make_golden.py (sinv_pair), written here
on device tensors.  Numerators 1e-10; Fisher, shot-noise, covariance and theory
contributions 1e-8; global and local sightlines, varying and constant masks, and S^-1
taken as its own transpose."""
import contextlib
import io
import os

import numpy as np
import pytest
import torch

from polybin3d_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def mask24(N, L):
    return synthetic.shell_mask(N, L, r_in=L / 6, r_out=0.4667 * L, n_holes=10, hole_r=(10.0, 30.0),
                                hole_box=0.4667 * L, seed=0)


def sinv_pair(base, N):
    """S^-1 x = IFT[w(k) FT[u x]], S^-dag x = u IFT[w(k) FT[x]] on device maps."""
    dev = base.device
    w = 1.0 / (1.0 + (torch.as_tensor(np.asarray(base.modk_grid), device=dev) / 0.05) ** 2)
    u = (1.0 + 0.5 * torch.sin(2 * np.pi * torch.arange(N, dtype=torch.float64, device=dev) / N))[:, None, None] \
        * torch.ones((N, N, N), dtype=torch.float64, device=dev)

    def sinv(x, input_type="real", output_type="real"):
        xr = base.to_real(x) if input_type == "fourier" else x
        y = base.to_fourier(u * xr) * w
        return y if output_type == "fourier" else base.to_real(y)

    def sinv_t(x, input_type="real", output_type="real"):
        X = x if input_type == "fourier" else base.to_fourier(x)
        yr = u * base.to_real(X * w)
        return base.to_fourier(yr) if output_type == "fourier" else yr
    return sinv, sinv_t


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLD, "custom_sinv.npz"))


def test_custom_sinv_global(g):
    import polybin3d_b200 as pb
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    pk_cov = [g["pk_k"], g["p0"], g["p2"]]
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="cuda")
    si, st = sinv_pair(b, N)
    ps = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=m, mask_shot=0.5 * m, applySinv=si, applySinv_transpose=st)
    assert rel(ps.Pk_numerator(d), g["a_num"]) < 1e-10
    assert rel(ps.compute_fisher_contribution(0), g["a_f0"]) < 1e-8
    assert rel(ps.compute_shot_contribution(1), g["a_s1"]) < 1e-8
    assert rel(ps.compute_covariance_contribution(2, pk_cov), g["a_c2"]) < 1e-8
    f, t = ps.compute_theory_contribution(3, g["kth"], lmax_theory=4)
    assert rel(f, g["a_f3"]) < 1e-8 and rel(t, g["a_t3"]) < 1e-8
    ps2 = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)), applySinv=si, applySinv_transpose=st)
    assert rel(ps2.Pk_numerator(synthetic.lognormal(N, L, seed=21).astype(np.float64) * 0.7), g["b_num"]) < 1e-10
    assert rel(ps2.compute_fisher_contribution(4), g["b_f4"]) < 1e-8
    assert rel(ps2.compute_covariance_contribution(5, pk_cov[:2]), g["b_c5"]) < 1e-8
    ps4 = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=m, applySinv=si)
    assert ps4.applySinv_transpose is si
    assert rel(ps4.compute_fisher_contribution(8), g["d_f8"]) < 1e-8


def test_custom_sinv_local(g):
    import polybin3d_b200 as pb
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=list(g["center"]), sightline="local", backend="cuda")
    si, st = sinv_pair(b, N)
    ps = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=m, mask_shot=0.5 * m, applySinv=si, applySinv_transpose=st)
    assert rel(ps.Pk_numerator(d), g["c_num"]) < 1e-10
    assert rel(ps.compute_fisher_contribution(6), g["c_f6"]) < 1e-8
    assert rel(ps.compute_shot_contribution(7), g["c_s7"]) < 1e-8


def test_custom_sinv_bispectrum():
    """BSpec with the caller's S^-1 (tests/golden/bk_custom_sinv.npz, lmax=2, CIC window):
    numerator without and with the linear term of generate_sims(2), Fisher, shot noise,
    covariance; and a constant mask."""
    import polybin3d_b200 as pb
    g = np.load(os.path.join(GOLD, "bk_custom_sinv.npz"))
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="cuda")
    si, st = sinv_pair(b, N)
    bs = quiet(pb.BSpec, b, g["edges"], lmax=2, mask=m, mask_shot=0.5 * m, applySinv=si, applySinv_transpose=st)
    assert np.array_equal(bs.all_bins, g["bins"])
    cub = quiet(bs.Bk_numerator, d, include_linear_term=False)
    assert rel(bs.sym_factor, g["sym"]) < 1e-12
    assert rel(cub, g["cub"]) < 1e-10
    quiet(bs.generate_sims, 2)
    num = quiet(bs.Bk_numerator, d)
    assert rel(num, g["num"]) < 1e-10 and rel(num - cub, g["num"] - g["cub"]) < 1e-8
    assert rel(quiet(bs.compute_fisher_contribution, 0), g["f0"]) < 1e-8
    assert rel(quiet(bs.compute_shot_contribution, 1, data=d, data2=0.7 * d), g["s1"]) < 1e-8
    assert rel(quiet(bs.compute_covariance_contribution, 2, [g["pk_k"], g["p0"], g["p2"]]), g["c2"]) < 1e-8
    bs2 = quiet(pb.BSpec, b, g["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)), applySinv=si, applySinv_transpose=st)
    d2 = synthetic.lognormal(N, L, seed=21).astype(np.float64) * 0.7
    assert rel(quiet(bs2.Bk_numerator, d2, include_linear_term=False), g["b_cub"]) < 1e-10
    assert rel(quiet(bs2.compute_fisher_contribution, 3), g["b_f3"]) < 1e-8
