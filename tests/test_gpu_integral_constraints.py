"""Integral constraints through the CUDA path against the reference's own outputs
(tests/golden/integral_constraints.npz, made by running the reference): the global
constraint (add_GIC) in the PSpec Fisher, covariance and theory contributions and in the
BSpec Fisher and covariance contributions and linear-term simulations; the radial
constraint (add_RIC, |r| shells, local sightline) in the PSpec and BSpec Fisher
contributions.  FP64: 1e-8 of the largest |entry| (Monte Carlo matrices), 1e-10 for the
numerator."""
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
    return np.load(os.path.join(GOLD, "integral_constraints.npz"))


def mask24(N, L):
    return synthetic.shell_mask(N, L, r_in=L / 6, r_out=0.4667 * L, n_holes=10, hole_r=(10.0, 30.0),
                                hole_box=0.4667 * L, seed=0)


def test_global_integral_constraint(g):
    import polybin3d_b200 as pb
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    mic = (m > 0).astype(np.float64)
    pk_cov = [g["pk_k"], g["p0"], g["p2"]]
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="cuda")
    ps = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=m, mask_shot=0.5 * m, add_GIC=True, mask_IC=mic)
    assert rel(ps.compute_fisher_contribution(0), g["pf0"]) < TOL
    assert rel(ps.compute_covariance_contribution(1, pk_cov), g["pc1"]) < TOL
    f, t = ps.compute_theory_contribution(2, g["kth"], lmax_theory=4)
    assert rel(f, g["pf2"]) < TOL and rel(t, g["pt2"]) < TOL
    bs = quiet(pb.BSpec, b, g["edges"], lmax=2, mask=m, mask_shot=0.5 * m, add_GIC=True, mask_IC=mic)
    assert np.array_equal(bs.all_bins, g["bins"])
    assert rel(quiet(bs.compute_fisher_contribution, 0), g["bf0"]) < TOL
    assert rel(quiet(bs.compute_covariance_contribution, 1, pk_cov), g["bc1"]) < TOL
    d = synthetic.lognormal(N, L, seed=13).astype(np.float64) * m
    quiet(bs.generate_sims, 2)
    num = quiet(bs.Bk_numerator, d)
    cub = quiet(bs.Bk_numerator, d, include_linear_term=False)
    assert rel(num, g["bnum"]) < 1e-10
    assert rel(num - cub, g["bnum"] - g["bcub"]) < TOL
    with pytest.raises(AssertionError):
        quiet(pb.PSpec, b, g["edges"], lmax=2, mask=m, add_GIC=True)
    with pytest.raises(AssertionError):
        quiet(pb.BSpec, b, g["edges"], lmax=2, mask=m, add_GIC=True, add_RIC=True, mask_IC=mic,
              radial_bins_RIC=[1.0, 2.0])


def test_radial_integral_constraint(g):
    import polybin3d_b200 as pb
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    mic = (m > 0).astype(np.float64)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="cuda", boxcenter=list(g["center"]),
              sightline="local")
    ps = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=m, add_RIC=True, mask_IC=mic, radial_bins_RIC=g["redges"])
    assert rel(ps.compute_fisher_contribution(3), g["lpf3"]) < TOL
    bs = quiet(pb.BSpec, b, g["edges"], lmax=2, mask=m, add_RIC=True, mask_IC=mic, radial_bins_RIC=g["redges"])
    assert rel(quiet(bs.compute_fisher_contribution, 2), g["lbf2"]) < TOL
