"""The bispectrum's linear term through the CUDA path: bias simulations from
generate_sims / load_sims and Bk_numerator(include_linear_term=True) against the
reference's own outputs (tests/golden/bk_linear.npz, made by running the reference), and
against the oracle at a size where the maps are synthesised on a dealiased grid.

FP64 mode meets 1e-10 on the numerator; the linear term alone (numerator minus the cubic
part, ~1e-5 of the numerator in case (a)) is held to 1e-8.  Mixed precision (FP32 maps,
tensor-core contraction) is held to 1e-5 of the largest |B| in a multipole block, on case
(c) where the linear term is of the order of the cubic part."""
import contextlib
import io
import os

import numpy as np
import pytest

from polybin3d_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


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
    return gold("bk_linear")


def make(pb, g, precision="fp64", lmax=2, mask=None, contraction="auto"):
    N, L = int(g["N"]), float(g["L"])
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision=precision)
    return quiet(pb.BSpec, b, g["edges"], lmax=lmax, mask=mask, contraction=contraction)


def test_generate_sims_varying_mask(pb, g):
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    bs = make(pb, g, mask=m)
    assert np.array_equal(bs.all_bins, g["bins"])
    quiet(bs.generate_sims, 3)
    d = synthetic.lognormal(N, L, seed=13).astype(np.float64) * m
    num = bs.Bk_numerator(d)
    cub = bs.Bk_numerator(d, include_linear_term=False)
    assert rel(cub, g["cub_a"]) < 1e-10
    assert rel(num, g["num_a"]) < 1e-10
    assert rel(num - cub, g["num_a"] - g["cub_a"]) < 1e-8


def test_generate_sims_constant_mask_tabulated_pk(pb, g):
    N, L = int(g["N"]), float(g["L"])
    bs = make(pb, g, lmax=0, mask=0.5 * np.ones((N, N, N)))
    assert bs.const_mask
    quiet(bs.generate_sims, 2, Pk_input=[g["pk_k"], g["pk_p"]])
    d = synthetic.lognormal(N, L, seed=14).astype(np.float64) * 0.5
    assert rel(bs.Bk_numerator(d), g["num_b"]) < 1e-10


@pytest.mark.parametrize("precision,contraction,tol", [("fp64", "auto", 1e-10), ("mixed", "simt", 1e-5),
                                                       ("mixed", "tc", 1e-5)])
def test_load_sims(pb, g, precision, contraction, tol):
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    bs = make(pb, g, precision=precision, mask=m, contraction=contraction)
    sims = [synthetic.grf(N, L, seed=60 + i) * m for i in range(2)]
    quiet(bs.load_sims, lambda ii: sims[ii], 2)
    d = synthetic.lognormal(N, L, seed=13).astype(np.float64) * m
    num = bs.Bk_numerator(d)
    nl = bs.N_bins // bs.Nl
    for j in range(bs.Nl):
        s = slice(j * nl, (j + 1) * nl)
        assert rel(num[s], g["num_c"][s]) < tol, j


def test_sims_fourier_input_and_no_preload(pb, g):
    """The same simulations given in Fourier space, and loaded lazily (preload=False),
    give the same numerator."""
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    sims = [synthetic.grf(N, L, seed=60 + i) * m for i in range(2)]
    d = synthetic.lognormal(N, L, seed=13).astype(np.float64) * m
    bs = make(pb, g, mask=m)
    quiet(bs.load_sims, lambda ii: np.fft.rfftn(sims[ii]), 2, input_type='fourier')
    assert rel(bs.Bk_numerator(d), g["num_c"]) < 1e-10
    bs2 = make(pb, g, mask=m)
    quiet(bs2.load_sims, lambda ii: sims[ii], 2, preload=False)
    assert rel(bs2.Bk_numerator(d), g["num_c"]) < 1e-10
    bs3 = make(pb, g, mask=m)
    quiet(bs3.generate_sims, 3, preload=False)
    assert rel(bs3.Bk_numerator(d), g["num_a"]) < 1e-10


def test_bk_unwindowed_with_linear_term(pb, g):
    """Bk_unwindowed's default include_linear_term=True, with a supplied Fisher."""
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    bs = make(pb, g, mask=m)
    quiet(bs.generate_sims, 3)
    d = synthetic.lognormal(N, L, seed=13).astype(np.float64) * m
    fish = np.diag(np.linspace(1.0, 2.0, bs.N_bins))
    out = quiet(bs.Bk_unwindowed, d, fish=fish)
    want = np.linalg.inv(fish) @ g["num_a"]
    nl = bs.N_bins // bs.Nl
    for j, l in enumerate(range(0, bs.lmax + 1, 2)):
        assert rel(out["b%d" % l], want[j * nl:(j + 1) * nl]) < 1e-10


def test_linear_term_dealiased_grid_against_oracle(pb):
    """48^3 with bins to 0.11 synthesises the data and simulation maps on a 32^3 grid;
    the linear term still matches the oracle's full-grid FP64 sums."""
    from oracle import polybin_oracle as O
    N, L = 48, 600.0
    edges = np.linspace(2 * np.pi / L, 0.11, 5)
    m = synthetic.shell_mask(N, L, r_in=L / 6, r_out=0.4667 * L, n_holes=10, hole_r=(10.0, 30.0),
                             hole_box=0.4667 * L, seed=0)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="cuda", precision="fp64")
    bs = quiet(pb.BSpec, b, edges, lmax=2, mask=m)
    assert tuple(bs.map_grid) != (N, N, N)
    sims = [synthetic.grf(N, L, seed=70 + i) * m for i in range(2)]
    quiet(bs.load_sims, lambda ii: sims[ii], 2)
    d = synthetic.lognormal(N, L, seed=15).astype(np.float64) * m
    num = bs.Bk_numerator(d)
    ob = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic")
    obs = O.OracleBSpec(ob, edges, lmax=2, mask=m)
    want = obs.numerator(d, "Sinv", sym=np.asarray(bs.sym_factor), sims=[obs.sim_spectrum(s) for s in sims])
    assert rel(num, want) < 1e-10
