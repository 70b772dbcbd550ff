"""Local (Yamamoto) line of sight through the CUDA path, against the reference's own outputs
(tests/golden/local_los.npz, made by running the reference with sightline='local'):
Pk (lmax=4) and Bk (lmax=2) numerators whose multipoles use the real harmonics of the voxel
positions and wavevectors, the symmetry factors, and the ideal (distant-observer) Fisher
matrices with mu measured from the direction of the box centre.  FP64 mode: 1e-10; mixed
precision: 1e-5 of the largest |value| of a multipole block."""
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
    return np.load(os.path.join(GOLD, "local_los.npz"))


def make_base(pb, g, precision="fp64"):
    N, L = int(g["N"]), float(g["L"])
    return quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=list(g["center"]), sightline="local",
                 pixel_window="cic", backend="cuda", precision=precision)


def blocks(a, b, n_blocks):
    nb = len(b) // n_blocks
    return max(rel(a[j * nb:(j + 1) * nb], b[j * nb:(j + 1) * nb]) for j in range(n_blocks))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_pk_local(pb, g, precision, tol):
    N, L = int(g["N"]), float(g["L"])
    b = make_base(pb, g, precision)
    m = mask24(N, L)
    ps = quiet(pb.PSpec, b, g["edges"], lmax=4, mask=m)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    assert blocks(ps.Pk_numerator_ideal(d), g["pk_num_ideal"], 3) < tol
    assert blocks(ps.Pk_numerator(d), g["pk_num"], 3) < tol
    pk = quiet(ps.Pk_ideal, d)
    assert rel(ps.fish_ideal, g["pk_fish_ideal"]) < 1e-10
    for k in ("p0", "p2", "p4"):
        assert rel(pk[k], g["Pk_" + k]) < (tol if precision == "fp64" else 1e-4), k


@pytest.mark.parametrize("precision,contraction,tol", [("fp64", "auto", 1e-10), ("mixed", "tc", 1e-5)])
def test_bk_local(pb, g, precision, contraction, tol):
    N, L = int(g["N"]), float(g["L"])
    b = make_base(pb, g, precision)
    m = mask24(N, L)
    bs = quiet(pb.BSpec, b, g["bedges"], lmax=2, mask=m, contraction=contraction)
    assert np.array_equal(bs.all_bins, g["bk_bins"])
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    num = quiet(bs.Bk_numerator_ideal, d)
    assert rel(bs.sym_factor, g["bk_sym"]) < 1e-10
    assert blocks(num, g["bk_num_ideal"], 2) < tol
    assert blocks(quiet(bs.Bk_numerator, d, include_linear_term=False), g["bk_num"], 2) < tol
    bk = quiet(bs.Bk_ideal, d)
    assert rel(bs.fish_ideal, g["bk_fish_ideal"]) < 1e-8
    for k in ("b0", "b2"):
        assert rel(bk[k], g["Bk_" + k]) < (tol if precision == "fp64" else 1e-4), k


def test_local_pk_fisher_contribution(pb):
    """Monte Carlo Pk Fisher contributions with the local line of sight on the reference's
    own noise (tests/golden/local_fisher.npz): varying and constant mask, lmax=4."""
    gf = np.load(os.path.join(GOLD, "local_fisher.npz"))
    N, L = int(gf["N"]), float(gf["L"])
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=list(gf["center"]), sightline="local",
              pixel_window="tsc", backend="cuda")
    ps = quiet(pb.PSpec, b, gf["edges"], lmax=4, mask=mask24(N, L))
    assert rel(ps.compute_fisher_contribution(0), gf["f0"]) < 1e-8
    ps2 = quiet(pb.PSpec, b, gf["edges"], lmax=4, mask=0.7 * np.ones((N, N, N)))
    assert rel(ps2.compute_fisher_contribution(1), gf["f1"]) < 1e-8


def test_local_bk_fisher_contribution(pb):
    """Monte Carlo Bk Fisher contributions (lmax=2) with the local line of sight on the
    reference's own noise pair: varying and constant mask."""
    gf = np.load(os.path.join(GOLD, "local_fisher.npz"))
    N, L = int(gf["N"]), float(gf["L"])
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=list(gf["center"]), sightline="local",
              pixel_window="tsc", backend="cuda")
    bs = quiet(pb.BSpec, b, gf["edges"], lmax=2, mask=mask24(N, L))
    assert np.array_equal(bs.all_bins, gf["bk_bins"])
    assert rel(quiet(bs.compute_fisher_contribution, 0), gf["bf0"]) < 1e-8
    bs2 = quiet(pb.BSpec, b, gf["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)))
    assert rel(quiet(bs2.compute_fisher_contribution, 1), gf["bf1"]) < 1e-8


def test_local_shot_noise(pb):
    """Shot-noise contributions with the local line of sight (PSpec lmax=4, BSpec lmax=2)
    against the reference's own outputs (tests/golden/local_shot.npz)."""
    gs = np.load(os.path.join(GOLD, "local_shot.npz"))
    N, L = int(gs["N"]), float(gs["L"])
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=[gs["pk_k"], gs["pk_p"]], boxcenter=list(gs["center"]),
              sightline="local", pixel_window="tsc", backend="cuda")
    m = mask24(N, L)
    ps = quiet(pb.PSpec, b, gs["edges"], lmax=4, mask=m, mask_shot=0.8 * m)
    assert rel(ps.compute_shot_contribution(1), gs["p_mask"]) < 1e-10
    bs = quiet(pb.BSpec, b, gs["edges"], lmax=2, mask=m, mask_shot=0.6 * m)
    assert np.array_equal(bs.all_bins, gs["bins"])
    d = synthetic.lognormal(N, L, seed=16).astype(np.float64) * m
    assert rel(quiet(bs.compute_shot_contribution, 1, data=d, data2=0.7 * d), gs["b_full"]) < 1e-10


def test_local_odd_multipoles(pb):
    """Odd multipoles of the local sightline (odd_l=True, lmax=3) and the wide-angle theory
    terms against the reference's outputs (tests/golden/local_odd.npz): S^-1 and ideal
    numerators (1e-10), Fisher, shot-noise and theory contributions (1e-8)."""
    go = np.load(os.path.join(GOLD, "local_odd.npz"))
    N, L = int(go["N"]), float(go["L"])
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=[go["pk_k"], go["pk_p"]], boxcenter=list(go["center"]),
              sightline="local", pixel_window="tsc", backend="cuda")
    m = mask24(N, L)
    ps = quiet(pb.PSpec, b, go["edges"], lmax=3, mask=m, mask_shot=0.8 * m, odd_l=True)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    assert blocks(ps.Pk_numerator(d), go["num"], 4) < 1e-10
    assert blocks(ps.Pk_numerator_ideal(d), go["num_ideal"], 2) < 1e-10
    assert rel(ps.compute_fisher_contribution(0), go["f0"]) < 1e-8
    assert rel(ps.compute_shot_contribution(1), go["shot1"]) < 1e-8
    f, t = ps.compute_theory_contribution(2, go["kth"], lmax_theory=4)
    assert rel(f, go["tf2"]) < 1e-8 and rel(t, go["tt2"]) < 1e-8
    pk = ps.Pk_unwindowed(d, fish=go["f0"])
    assert sorted(pk) == ["p0", "p1", "p2", "p3"]
    ps2 = quiet(pb.PSpec, b, go["edges"], lmax=2, mask=m)
    f, t = ps2.compute_theory_contribution(3, go["kth"], lmax_theory=4, include_wideangle=True)
    assert rel(f, go["wf3"]) < 1e-8 and rel(t, go["wt3"]) < 1e-8
    with pytest.raises(AssertionError):
        ps.compute_theory_contribution(2, go["kth"], lmax_theory=4, include_wideangle=True)


def test_base_harmonic_transforms(pb):
    """PolyBin3D.apply_fourier_harmonics / apply_real_harmonics / apply_xi with the harmonic
    grids PSpec keeps in Ylm_real / Ylm_fourier, against the oracle's restatement of
    base.py:391-437 (local sightline, l = 2 and 4, Pk_grid with three multipoles)."""
    from oracle import polybin_oracle as O
    N, L = 24, 600.0
    center = [700.0, 400.0, 900.0]
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=center, sightline="local", backend="cuda")
    ps = quiet(pb.PSpec, b, np.linspace(2 * np.pi / L, 0.11, 5), lmax=4)
    assert sorted(ps.Ylm_real) == [2, 4] and sorted(ps.Ylm_fourier) == [2, 4]
    ob = O.OracleBase([L] * 3, [N] * 3, boxcenter=np.asarray(center), sightline="local")
    x = synthetic.lognormal(N, L, seed=5).astype(np.float64)
    X = ob.to_fourier(x)
    for l in (2, 4):
        got = b.apply_fourier_harmonics(x, ps.Ylm_real[l], ps.Ylm_fourier[l]).cpu().numpy()
        assert rel(got, ob.apply_fourier_harmonics(x, l)) < 1e-12
        got = b.apply_real_harmonics(X, ps.Ylm_real[l], ps.Ylm_fourier[l]).cpu().numpy()
        assert rel(got, ob.apply_real_harmonics(X, l)) < 1e-12
    kt = np.linspace(0.0, 1.0, 500)
    pk_cov = [kt, 3e3 * np.exp(-(kt / 0.25) ** 2), 800.0 * np.exp(-(kt / 0.2) ** 2), 100.0 * np.exp(-kt / 0.2)]
    xi = O.xi_grids(ob, pk_cov)
    for out in ("real", "fourier"):
        got = b.apply_xi(X, x, ps.Ylm_real, ps.Ylm_fourier, xi, output_type=out).cpu().numpy()
        assert rel(got, O.apply_xi(ob, X, x, xi, out)) < 1e-12
