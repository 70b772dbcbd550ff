"""Covariance and theory-matrix Monte Carlo contributions of PSpec through the CUDA path,
against the reference's own outputs on its own noise (tests/golden/pk_cov_theory.npz, made
by running the reference): global sightline with lmax=4 (Pk_cov = [k, P0, P2] with a varying
mask and mask_shot, and a constant mask; theory matrix with lmax_theory = 4 in 6 theory
bins), local sightline with lmax=2 (covariance with [k, P0, P2] and with [k, P0] for a
constant mask; theory matrix with lmax_theory = 4).  FP64 throughout: 1e-8 of the largest
|entry|, the Monte Carlo Fisher tolerance."""
import contextlib
import io
import os

import numpy as np
import pytest

from polybin3d_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-8


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLD, "pk_cov_theory.npz"))


def mask24(N, L):
    return synthetic.shell_mask(N, L, r_in=L / 6, r_out=0.4667 * L, n_holes=10, hole_r=(10.0, 30.0),
                                hole_box=0.4667 * L, seed=0)


def test_covariance_global(g):
    import polybin3d_b200 as pb
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    pk_cov = [g["pk_k"], g["p0"], g["p2"]]
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="cuda")
    ps = quiet(pb.PSpec, b, g["edges"], lmax=4, mask=m, mask_shot=0.5 * m)
    assert rel(ps.compute_covariance_contribution(2, pk_cov), g["c2"]) < TOL
    ps2 = quiet(pb.PSpec, b, g["edges"], lmax=4, mask=0.7 * np.ones((N, N, N)))
    assert rel(ps2.compute_covariance_contribution(3, pk_cov), g["c3"]) < TOL
    with pytest.raises(AssertionError):
        quiet(pb.PSpec, b, g["edges"], lmax=0, mask=m, mask_shot=m).compute_covariance_contribution(0, pk_cov)


def test_theory_global(g):
    import polybin3d_b200 as pb
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="cuda")
    ps = quiet(pb.PSpec, b, g["edges"], lmax=4, mask=m, mask_shot=0.5 * m)
    f, t = ps.compute_theory_contribution(4, g["kth"], lmax_theory=4)
    assert t.shape == g["t4"].shape
    assert rel(f, g["f4"]) < TOL and rel(t, g["t4"]) < TOL
    with pytest.raises(AssertionError):
        ps.compute_theory_contribution(4, np.linspace(0.01, 0.2, 5))
    with pytest.raises(AssertionError):
        ps.compute_theory_contribution(4, g["kth"], include_wideangle=True)


def test_covariance_theory_local(g):
    import polybin3d_b200 as pb
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    pk_cov = [g["pk_k"], g["p0"], g["p2"]]
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", boxcenter=list(g["center"]),
              sightline="local")
    ps = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=m, mask_shot=0.5 * m)
    assert rel(ps.compute_covariance_contribution(5, pk_cov), g["lc5"]) < TOL
    f, t = ps.compute_theory_contribution(6, g["kth"], lmax_theory=4)
    assert rel(f, g["lf6"]) < TOL and rel(t, g["lt6"]) < TOL
    ps2 = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)))
    assert rel(ps2.compute_covariance_contribution(7, pk_cov[:2]), g["lc7"]) < TOL
    with pytest.raises(ValueError):
        ps2.compute_covariance_contribution(7, pk_cov)


def test_bk_covariance():
    """BSpec covariance contributions (lmax=2, tests/golden/bk_cov.npz): global sightline
    with the bispectrum's shot mask and with a separate two-point one, constant mask, and
    the local sightline."""
    import polybin3d_b200 as pb
    gb = np.load(os.path.join(GOLD, "bk_cov.npz"))
    N, L = int(gb["N"]), float(gb["L"])
    m = mask24(N, L)
    pk_cov = [gb["pk_k"], gb["p0"], gb["p2"]]
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="cuda")
    bs = quiet(pb.BSpec, b, gb["edges"], lmax=2, mask=m, mask_shot=0.5 * m)
    assert np.array_equal(bs.all_bins, gb["bins"])
    assert rel(quiet(bs.compute_covariance_contribution, 2, pk_cov), gb["c2"]) < TOL
    assert rel(quiet(bs.compute_covariance_contribution, 3, pk_cov, mask_shot_2pt=0.8 * m), gb["c3"]) < TOL
    bs2 = quiet(pb.BSpec, b, gb["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)))
    assert rel(quiet(bs2.compute_covariance_contribution, 4, pk_cov[:2]), gb["c4"]) < TOL
    lb = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", boxcenter=list(gb["center"]),
               sightline="local")
    lbs = quiet(pb.BSpec, lb, gb["edges"], lmax=2, mask=m, mask_shot=0.5 * m)
    assert rel(quiet(lbs.compute_covariance_contribution, 5, pk_cov), gb["lc5"]) < TOL
