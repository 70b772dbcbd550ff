"""Shot-noise Monte Carlo through the CUDA path: PSpec.compute_shot_contribution and
BSpec.compute_shot_contribution (quadratic and cubic terms) against the reference's own
outputs (tests/golden/shot.npz, made by running the reference) in FP64 mode (1e-10), and in
mixed precision (FP32 maps, tensor-core contraction) to 1e-5 of the largest |value| in a
multipole block; the subtraction in Pk_unwindowed."""
import contextlib
import io
import os

import numpy as np
import pytest

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


@pytest.fixture(scope="module")
def pb():
    import polybin3d_b200
    return polybin3d_b200


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(GOLD, "shot.npz"))


def make_base(pb, g, precision="fp64"):
    N, L = int(g["N"]), float(g["L"])
    return quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=[g["pk_k"], g["pk_p"]], pixel_window="tsc", backend="cuda",
                 precision=precision)


def test_pk_shot(pb, g):
    N, L = int(g["N"]), float(g["L"])
    b = make_base(pb, g)
    m = mask24(N, L)
    ps = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=m, mask_shot=0.8 * m)
    assert rel(ps.compute_shot_contribution(1), g["p_mask"]) < 1e-10
    ps2 = quiet(pb.PSpec, b, g["edges"], lmax=2)
    assert rel(ps2.compute_shot_contribution(2), g["p_nomask"]) < 1e-10


def test_pk_unwindowed_subtracts_shot(pb, g):
    N, L = int(g["N"]), float(g["L"])
    b = make_base(pb, g)
    m = mask24(N, L)
    ps = quiet(pb.PSpec, b, g["edges"], lmax=2, mask=m, mask_shot=0.8 * m)
    fish = np.diag(np.linspace(1.0, 3.0, ps.N_bins))
    shot = ps.compute_shot_contribution(1)
    d = synthetic.lognormal(N, L, seed=16).astype(np.float64) * m
    out = quiet(ps.Pk_unwindowed, d, fish=fish, shot_num=shot, subtract_shotnoise=True)
    want = np.linalg.inv(fish) @ (ps.Pk_numerator(d) - shot)
    for li in range(ps.Nl):
        assert rel(out["p%d" % (2 * li)], want[li * ps.Nk:(li + 1) * ps.Nk]) < 1e-12


@pytest.mark.parametrize("precision,contraction,tol", [("fp64", "auto", 1e-10), ("mixed", "tc", 1e-5),
                                                       ("mixed", "simt", 1e-5)])
def test_bk_shot(pb, g, precision, contraction, tol):
    N, L = int(g["N"]), float(g["L"])
    b = make_base(pb, g, precision)
    m = mask24(N, L)
    bs = quiet(pb.BSpec, b, g["edges"], lmax=2, mask=m, mask_shot=0.6 * m, contraction=contraction)
    assert np.array_equal(bs.all_bins, g["bins"])
    d = synthetic.lognormal(N, L, seed=16).astype(np.float64) * m
    full = quiet(bs.compute_shot_contribution, 1, data=d, data2=0.7 * d)
    cub = quiet(bs.compute_shot_contribution, 1, cubic_only=True)
    nl = bs.N_bins // bs.Nl
    for j in range(bs.Nl):
        s = slice(j * nl, (j + 1) * nl)
        assert rel(full[s], g["b_full"][s]) < tol, j
        assert rel(cub[s], g["b_cubic"][s]) < tol, j


def test_bk_shot_needs_data_and_mask_shot(pb, g):
    N, L = int(g["N"]), float(g["L"])
    b = make_base(pb, g)
    bs = quiet(pb.BSpec, b, g["edges"], lmax=0)
    with pytest.raises(AssertionError, match="Must supply data"):
        bs.compute_shot_contribution(0)
    with pytest.raises(AssertionError, match="triply-weighted mask"):
        quiet(bs.compute_shot_contribution, 0, cubic_only=True)
