"""Pin the oracle to the reference: every golden fixture (made by running the reference,
tests/golden/make_golden.py) is reproduced by oracle/polybin_oracle.py."""
import os

import numpy as np
import pytest

from oracle import polybin_oracle as O
from polybin3d_b200 import synthetic

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-11


def gold(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def field(g):
    kind, seed, N, L = str(g["data_kind"]), int(g["data_seed"]), int(g["N"]), float(g["L"])
    return synthetic.grf(N, L, seed) if kind == "grf" else synthetic.lognormal(N, L, seed)


def mask24(N, L):
    return synthetic.shell_mask(N, L, r_in=L / 6, r_out=0.4667 * L, n_holes=10, hole_r=(10.0, 30.0),
                                hole_box=0.4667 * L, seed=0)


def test_cfg1_pk_bk():
    g = gold("cfg1")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3)
    d = field(g)
    ps = O.OraclePSpec(b, g["edges"], lmax=2)
    assert rel(ps.numerator(d), g["pk_num"]) < TOL
    assert rel(ps.fisher_ideal(), g["pk_fish"]) < TOL
    pk = ps.Pk_ideal(d)
    for k in pk:
        assert rel(pk[k], g["Pk_" + k]) < TOL
    bs = O.OracleBSpec(b, g["edges"], lmax=0)
    assert np.array_equal(bs.all_bins, g["bk_bins"])
    sym = bs.symmetry_factor()
    assert np.array_equal(sym, g["bk_sym"])
    assert rel(bs.numerator(d, sym=sym), g["bk_num"]) < TOL
    assert rel(bs.fisher_ideal(sym=sym), g["bk_fish"]) < TOL
    bk = bs.Bk_ideal(d, sym=sym)
    assert rel(bk["b0"], g["Bk_b0"]) < TOL


def test_bk_lmax2_tsc():
    g = gold("bk_l2_tsc")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="tsc")
    bs = O.OracleBSpec(b, g["edges"], lmax=2)
    assert np.array_equal(bs.all_bins, g["bk_bins"])
    sym = bs.symmetry_factor()
    assert rel(sym, g["bk_sym"]) < TOL
    d = field(g)
    assert rel(bs.numerator(d, sym=sym), g["bk_num"]) < TOL
    assert rel(bs.fisher_ideal(sym=sym), g["bk_fish"]) < TOL
    assert rel(bs.fisher_ideal(False, sym=sym), g["bk_fish_nodisc"]) < TOL
    bk = bs.Bk_ideal(d, sym=sym)
    for k in bk:
        assert rel(bk[k], g["Bk_" + k]) < TOL


def test_bk_squeezed_partial_triangles():
    g = gold("bk_squeeze_partial")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic")
    bs = O.OracleBSpec(b, g["edges"], lmax=0, k_bins_squeeze=g["edges_sq"], include_partial_triangles=True)
    assert np.array_equal(bs.all_bins, g["bk_bins"])
    d = field(g)
    sym = bs.symmetry_factor()
    assert rel(bs.numerator(d, sym=sym), g["bk_num"]) < TOL
    bk = bs.Bk_ideal(d, sym=sym)
    assert rel(bk["b0"], g["Bk_b0"]) < TOL


@pytest.mark.parametrize("pw", ["cic", "interlaced-tsc"])
def test_pk_windows_tabulated_pk(pw):
    g = gold("pk_windows")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, Pk=synthetic.pk_table(1.0), pixel_window=pw)
    ps = O.OraclePSpec(b, g["edges"], lmax=4)
    d = field(g)
    tag = pw.replace("-", "_")
    assert rel(ps.numerator(d), g[tag + "_num"]) < TOL
    assert rel(ps.fisher_ideal(), g[tag + "_fish"]) < TOL
    assert rel(ps.fisher_ideal(False), g[tag + "_fish_nodisc"]) < TOL


def test_grf_from_reference_noise():
    g = gold("grf_noise")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, Pk=synthetic.pk_table(1.0), pixel_window="cic")
    assert rel(b.grf_from_noise(*b.reference_noise(int(g["seed"]))), g["a"]) < 1e-14


def test_pk_fisher_masked_and_qmaps():
    g = gold("pk_fisher_mask")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3)
    ps = O.OraclePSpec(b, g["edges"], lmax=4, mask=mask24(N, L))
    f0 = ps.fisher_contribution(b.reference_noise(0 + 10 ** 7))
    f1 = ps.fisher_contribution(b.reference_noise(1 + 10 ** 7))
    assert rel(f0, g["f0"]) < TOL and rel(f1, g["f1"]) < TOL


def test_pk_fisher_nomask():
    g = gold("pk_fisher_nomask")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="tsc")
    ps = O.OraclePSpec(b, g["edges"], lmax=2)
    assert rel(ps.fisher_contribution(b.reference_noise(2 + 10 ** 7)), g["f2"]) < TOL


def test_bk_fisher_masked_and_qmaps():
    g = gold("bk_fisher_mask")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3)
    m = mask24(N, L)
    bs = O.OracleBSpec(b, g["edges"], lmax=0, mask=m)
    assert np.array_equal(bs.all_bins, g["bins0"])
    f, Q = bs.fisher_contribution(b.reference_noise(10 ** 7), b.reference_noise(2 * 10 ** 7), return_Q=True)
    assert rel(f, g["f0"]) < TOL
    assert rel(Q, g["q0"]) < TOL
    bs2 = O.OracleBSpec(b, g["edges"], lmax=2, mask=m)
    f2 = bs2.fisher_contribution(b.reference_noise(10 ** 7), b.reference_noise(2 * 10 ** 7))
    assert rel(f2, g["f2_l2"]) < TOL


def test_bk_fisher_nomask_lmax2():
    g = gold("bk_fisher_nomask")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic")
    bs = O.OracleBSpec(b, g["edges"], lmax=2)
    assert rel(bs.symmetry_factor(), g["sym"]) < TOL
    f = bs.fisher_contribution(b.reference_noise(3 + 10 ** 7), b.reference_noise(3 + 2 * 10 ** 7))
    assert rel(f, g["f3"]) < TOL


def test_bk_linear_term():
    """Bk_numerator with the linear term: generate_sims under a varying mask (a) and a
    constant mask with a tabulated P(k) (b), load_sims of real-space maps (c).  The linear
    term itself (numerator minus the cubic part) is checked on its own in (a): it is ~1e-5
    of the numerator there."""
    from scipy.interpolate import interp1d
    g = gold("bk_linear")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="tsc")
    m = mask24(N, L)
    d = synthetic.lognormal(N, L, seed=13).astype(np.float64) * m
    bs = O.OracleBSpec(b, g["edges"], lmax=2, mask=m)
    assert np.array_equal(bs.all_bins, g["bins"])
    sym = g["sym"]
    sims = [bs.generated_sim(i) for i in range(3)]
    num = bs.numerator(d, "Sinv", sym=sym, sims=sims)
    cub = bs.numerator(d, "Sinv", sym=sym)
    assert rel(cub, g["cub_a"]) < TOL
    assert rel(num, g["num_a"]) < TOL
    assert rel(num - cub, g["num_a"] - g["cub_a"]) < 1e-8
    # (b)
    bs2 = O.OracleBSpec(b, g["edges"], lmax=0, mask=0.5 * np.ones((N, N, N)))
    assert bs2.const_mask
    pk = interp1d(g["pk_k"], g["pk_p"], bounds_error=False, fill_value=0.)(b.modk_grid)
    d2 = synthetic.lognormal(N, L, seed=14).astype(np.float64) * 0.5
    sims2 = [bs2.generated_sim(i, Pk_grid=pk) for i in range(2)]
    assert rel(bs2.numerator(d2, "Sinv", sims=sims2), g["num_b"]) < TOL
    # (c)
    sims3 = [bs.sim_spectrum(synthetic.grf(N, L, seed=60 + i) * m) for i in range(2)]
    assert rel(bs.numerator(d, "Sinv", sym=sym, sims=sims3), g["num_c"]) < TOL


def test_shot_noise():
    """compute_shot_contribution of PSpec (masked and unmasked) and BSpec (full and cubic
    only), tabulated fiducial spectrum, TSC window."""
    g = gold("shot")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, Pk=[g["pk_k"], g["pk_p"]], pixel_window="tsc")
    m = mask24(N, L)
    ps = O.OraclePSpec(b, g["edges"], lmax=2, mask=m)
    assert rel(ps.shot_contribution(b.reference_noise(1 + 10 ** 7), mask_shot=0.8 * m), g["p_mask"]) < TOL
    ps2 = O.OraclePSpec(b, g["edges"], lmax=2)
    assert rel(ps2.shot_contribution(b.reference_noise(2 + 10 ** 7)), g["p_nomask"]) < TOL
    bs = O.OracleBSpec(b, g["edges"], lmax=2, mask=m)
    assert np.array_equal(bs.all_bins, g["bins"])
    n1, n2 = b.reference_noise(1 + 10 ** 7), b.reference_noise(1 + 2 * 10 ** 7)
    d = synthetic.lognormal(N, L, seed=16).astype(np.float64) * m
    assert rel(bs.shot_contribution(n1, n2, 0.6 * m, cubic_only=True, sym=g["sym"]), g["b_cubic"]) < TOL
    assert rel(bs.shot_contribution(n1, n2, 0.6 * m, data=d, data2=0.7 * d, sym=g["sym"]), g["b_full"]) < TOL


def test_local_line_of_sight():
    """Pk and Bk with the local (Yamamoto) line of sight: multipoles of the numerators through
    the real harmonics of positions and wavevectors; the ideal Fisher matrices are the
    distant-observer ones with mu measured from the direction of the box centre."""
    g = gold("local_los")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic", boxcenter=g["center"], sightline="local")
    m = mask24(N, L)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    ps = O.OraclePSpec(b, g["edges"], lmax=4, mask=m)
    assert rel(ps.numerator(d, "ideal"), g["pk_num_ideal"]) < TOL
    assert rel(ps.numerator(d, "Sinv"), g["pk_num"]) < TOL
    assert rel(ps.fisher_ideal(), g["pk_fish_ideal"]) < TOL
    pk = ps.Pk_ideal(d)
    for k in ("p0", "p2", "p4"):
        assert rel(pk[k], g["Pk_" + k]) < TOL
    bs = O.OracleBSpec(b, g["bedges"], lmax=2, mask=m)
    assert np.array_equal(bs.all_bins, g["bk_bins"])
    assert rel(bs.symmetry_factor(), g["bk_sym"]) < TOL
    assert rel(bs.numerator(d, "ideal", sym=g["bk_sym"]), g["bk_num_ideal"]) < TOL
    assert rel(bs.numerator(d, "Sinv", sym=g["bk_sym"]), g["bk_num"]) < TOL
    assert rel(bs.fisher_ideal(sym=g["bk_sym"]), g["bk_fish_ideal"]) < TOL
    bk = bs.Bk_ideal(d, sym=g["bk_sym"])
    for k in ("b0", "b2"):
        assert rel(bk[k], g["Bk_" + k]) < TOL


def test_local_fisher_contribution():
    """Monte Carlo Pk and Bk Fisher contributions with the local line of sight (varying and
    constant mask), on the reference's own noise."""
    g = gold("local_fisher")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="tsc", boxcenter=g["center"], sightline="local")
    ps = O.OraclePSpec(b, g["edges"], lmax=4, mask=mask24(N, L))
    assert rel(ps.fisher_contribution(b.reference_noise(0 + 10 ** 7)), g["f0"]) < TOL
    ps2 = O.OraclePSpec(b, g["edges"], lmax=4, mask=0.7 * np.ones((N, N, N)))
    assert rel(ps2.fisher_contribution(b.reference_noise(1 + 10 ** 7)), g["f1"]) < TOL
    bs = O.OracleBSpec(b, g["edges"], lmax=2, mask=mask24(N, L))
    assert np.array_equal(bs.all_bins, g["bk_bins"])
    f = bs.fisher_contribution(b.reference_noise(10 ** 7), b.reference_noise(2 * 10 ** 7), sym=g["bk_sym"])
    assert rel(f, g["bf0"]) < TOL
    bs2 = O.OracleBSpec(b, g["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)))
    f = bs2.fisher_contribution(b.reference_noise(1 + 10 ** 7), b.reference_noise(1 + 2 * 10 ** 7), sym=g["bk_sym"])
    assert rel(f, g["bf1"]) < TOL


def test_local_shot_noise():
    """Shot-noise contributions with the local line of sight (PSpec lmax=4, BSpec lmax=2)."""
    g = gold("local_shot")
    N, L = int(g["N"]), float(g["L"])
    b = O.OracleBase([L] * 3, [N] * 3, Pk=[g["pk_k"], g["pk_p"]], pixel_window="tsc", boxcenter=g["center"],
                     sightline="local")
    m = mask24(N, L)
    ps = O.OraclePSpec(b, g["edges"], lmax=4, mask=m)
    assert rel(ps.shot_contribution(b.reference_noise(1 + 10 ** 7), mask_shot=0.8 * m), g["p_mask"]) < TOL
    bs = O.OracleBSpec(b, g["edges"], lmax=2, mask=m)
    assert np.array_equal(bs.all_bins, g["bins"])
    n1, n2 = b.reference_noise(1 + 10 ** 7), b.reference_noise(1 + 2 * 10 ** 7)
    d = synthetic.lognormal(N, L, seed=16).astype(np.float64) * m
    assert rel(bs.shot_contribution(n1, n2, 0.6 * m, data=d, data2=0.7 * d, sym=g["sym"]), g["b_full"]) < TOL


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors of the Random123 distribution (kat_vectors)."""
    cases = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
             ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
             ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
              (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for c, k, want in cases:
        got = O.philox4x32_10(*[np.array([v], dtype=np.uint64) for v in c], *k)
        assert [int(g[0]) for g in got] == list(want)


def test_philox_noise_is_gaussian():
    b = O.OracleBase([500.0] * 3, [32] * 3)
    re, im = b.philox_noise(12345)
    x = np.concatenate([re.ravel(), im.ravel()])
    assert abs(x.mean()) < 5e-3 and abs(x.std() - 1) < 5e-3
    re2, _ = b.philox_noise(12346)
    assert abs(np.corrcoef(re.ravel(), re2.ravel())[0, 1]) < 5e-3


def test_pk_covariance_and_theory():
    """Covariance (Pk_cov with P0, P2; varying mask with mask_shot, constant mask) and theory
    matrix contributions (lmax_theory = 4), global and local sightlines, on the reference's
    own noise."""
    g = gold("pk_cov_theory")
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    pk_cov = [g["pk_k"], g["p0"], g["p2"]]
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic")
    ps = O.OraclePSpec(b, g["edges"], lmax=4, mask=m)
    assert rel(ps.covariance_contribution(b.reference_noise(2 + 10 ** 7), pk_cov, mask_shot=0.5 * m), g["c2"]) < TOL
    ps2 = O.OraclePSpec(b, g["edges"], lmax=4, mask=0.7 * np.ones((N, N, N)))
    assert rel(ps2.covariance_contribution(b.reference_noise(3 + 10 ** 7), pk_cov), g["c3"]) < TOL
    f, t = ps.theory_contribution(b.reference_noise(4 + 10 ** 7), g["kth"], lmax_theory=4)
    assert rel(f, g["f4"]) < TOL and rel(t, g["t4"]) < TOL
    lb = O.OracleBase([L] * 3, [N] * 3, pixel_window="tsc", boxcenter=g["center"], sightline="local")
    lps = O.OraclePSpec(lb, g["edges"], lmax=2, mask=m)
    assert rel(lps.covariance_contribution(lb.reference_noise(5 + 10 ** 7), pk_cov, mask_shot=0.5 * m),
               g["lc5"]) < TOL
    f, t = lps.theory_contribution(lb.reference_noise(6 + 10 ** 7), g["kth"], lmax_theory=4)
    assert rel(f, g["lf6"]) < TOL and rel(t, g["lt6"]) < TOL
    lps2 = O.OraclePSpec(lb, g["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)))
    assert rel(lps2.covariance_contribution(lb.reference_noise(7 + 10 ** 7), pk_cov[:2]), g["lc7"]) < TOL


def test_bk_covariance():
    """BSpec covariance contributions (lmax=2, Pk_cov with P0, P2): global sightline with the
    shared and a separate two-point shot mask, constant mask, local sightline."""
    g = gold("bk_cov")
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    pk_cov = [g["pk_k"], g["p0"], g["p2"]]
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic")
    bs = O.OracleBSpec(b, g["edges"], lmax=2, mask=m)
    assert np.array_equal(bs.all_bins, g["bins"])
    sym = g["sym"]
    n = lambda s: (b.reference_noise(s + 10 ** 7), b.reference_noise(s + 2 * 10 ** 7))
    assert rel(bs.covariance_contribution(*n(2), pk_cov, mask_shot_2pt=0.5 * m, sym=sym), g["c2"]) < TOL
    assert rel(bs.covariance_contribution(*n(3), pk_cov, mask_shot_2pt=0.8 * m, sym=sym), g["c3"]) < TOL
    bs2 = O.OracleBSpec(b, g["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)))
    assert rel(bs2.covariance_contribution(*n(4), pk_cov[:2], sym=sym), g["c4"]) < TOL
    lb = O.OracleBase([L] * 3, [N] * 3, pixel_window="tsc", boxcenter=g["center"], sightline="local")
    lbs = O.OracleBSpec(lb, g["edges"], lmax=2, mask=m)
    ln = (lb.reference_noise(5 + 10 ** 7), lb.reference_noise(5 + 2 * 10 ** 7))
    assert rel(lbs.covariance_contribution(*ln, pk_cov, mask_shot_2pt=0.5 * m, sym=g["lsym"]), g["lc5"]) < TOL


def test_integral_constraints():
    """Global (GIC) and radial (RIC) integral constraints in the pointing matrix of the Monte
    Carlo Fisher, covariance and theory matrices and of the linear term's simulations."""
    g = gold("integral_constraints")
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    mic = (m > 0).astype(np.float64)
    pk_cov = [g["pk_k"], g["p0"], g["p2"]]
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic")
    ps = O.OraclePSpec(b, g["edges"], lmax=2, mask=m, mask_IC=mic, add_GIC=True)
    assert rel(ps.fisher_contribution(b.reference_noise(10 ** 7)), g["pf0"]) < TOL
    assert rel(ps.covariance_contribution(b.reference_noise(1 + 10 ** 7), pk_cov, mask_shot=0.5 * m), g["pc1"]) < TOL
    f, t = ps.theory_contribution(b.reference_noise(2 + 10 ** 7), g["kth"], lmax_theory=4)
    assert rel(f, g["pf2"]) < TOL and rel(t, g["pt2"]) < TOL
    bs = O.OracleBSpec(b, g["edges"], lmax=2, mask=m, mask_IC=mic, add_GIC=True)
    assert np.array_equal(bs.all_bins, g["bins"])
    sym = g["sym"]
    n = lambda s, bb: (bb.reference_noise(s + 10 ** 7), bb.reference_noise(s + 2 * 10 ** 7))
    assert rel(bs.fisher_contribution(*n(0, b), sym=sym), g["bf0"]) < TOL
    assert rel(bs.covariance_contribution(*n(1, b), pk_cov, mask_shot_2pt=0.5 * m, sym=sym), g["bc1"]) < TOL
    d = synthetic.lognormal(N, L, seed=13).astype(np.float64) * m
    sims = [bs.generated_sim(i) for i in range(2)]
    num = bs.numerator(d, "Sinv", sym=sym, sims=sims)
    cub = bs.numerator(d, "Sinv", sym=sym)
    assert rel(num, g["bnum"]) < TOL and rel(cub, g["bcub"]) < TOL
    assert rel(num - cub, g["bnum"] - g["bcub"]) < 1e-8
    lb = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic", boxcenter=g["center"], sightline="local")
    lps = O.OraclePSpec(lb, g["edges"], lmax=2, mask=m, mask_IC=mic, add_RIC=True, radial_bins_RIC=g["redges"])
    assert rel(lps.fisher_contribution(lb.reference_noise(3 + 10 ** 7)), g["lpf3"]) < TOL
    lbs = O.OracleBSpec(lb, g["edges"], lmax=2, mask=m, mask_IC=mic, add_RIC=True, radial_bins_RIC=g["redges"])
    assert rel(lbs.fisher_contribution(*n(2, lb), sym=g["lsym"]), g["lbf2"]) < TOL


def test_local_odd_multipoles():
    """Odd multipoles of the local sightline (odd_l, lmax=3): numerators, Fisher, shot noise
    and theory matrix; and the wide-angle theory terms (lmax=2, lmax_theory=4)."""
    g = gold("local_odd")
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    b = O.OracleBase([L] * 3, [N] * 3, Pk=[g["pk_k"], g["pk_p"]], pixel_window="tsc", boxcenter=g["center"],
                     sightline="local")
    ps = O.OraclePSpec(b, g["edges"], lmax=3, mask=m, odd_l=True)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    assert rel(ps.numerator(d, "Sinv"), g["num"]) < TOL
    assert rel(ps.numerator(d, "ideal"), g["num_ideal"]) < TOL
    assert rel(ps.fisher_contribution(b.reference_noise(10 ** 7)), g["f0"]) < TOL
    assert rel(ps.shot_contribution(b.reference_noise(1 + 10 ** 7), mask_shot=0.8 * m), g["shot1"]) < TOL
    f, t = ps.theory_contribution(b.reference_noise(2 + 10 ** 7), g["kth"], lmax_theory=4)
    assert rel(f, g["tf2"]) < TOL and rel(t, g["tt2"]) < TOL
    ps2 = O.OraclePSpec(b, g["edges"], lmax=2, mask=m)
    f, t = ps2.theory_contribution(b.reference_noise(3 + 10 ** 7), g["kth"], lmax_theory=4, include_wideangle=True)
    assert rel(f, g["wf3"]) < TOL and rel(t, g["wt3"]) < TOL


def sinv_pair(base, N):
    """The fixture's S^-1 = IFT w(k) FT u and its transpose u IFT w(k) FT (make_golden.sinv_pair)."""
    w = 1.0 / (1.0 + (np.asarray(base.modk_grid) / 0.05) ** 2)
    u = (1.0 + 0.5 * np.sin(2 * np.pi * np.arange(N) / N))[:, None, None] * np.ones((N, N, N))

    def sinv(x, input_type="real", output_type="real"):
        xr = base.to_real(x) if input_type == "fourier" else x
        y = base.to_fourier(u * xr) * w
        return y if output_type == "fourier" else base.to_real(y)

    def sinv_t(x, input_type="real", output_type="real"):
        X = x if input_type == "fourier" else base.to_fourier(x)
        yr = u * base.to_real(X * w)
        return base.to_fourier(yr) if output_type == "fourier" else yr
    return sinv, sinv_t


def test_custom_sinv():
    """A caller's S^-1 (and S^-dag) in the numerator, Fisher, shot-noise, covariance and
    theory contributions; global and local sightlines, varying and constant masks."""
    g = gold("custom_sinv")
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    pk_cov = [g["pk_k"], g["p0"], g["p2"]]
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic")
    si, st = sinv_pair(b, N)
    ps = O.OraclePSpec(b, g["edges"], lmax=2, mask=m, applySinv=si, applySinv_transpose=st)
    n = lambda s, bb: bb.reference_noise(s + 10 ** 7)
    assert rel(ps.numerator(d, "Sinv"), g["a_num"]) < TOL
    assert rel(ps.fisher_contribution(n(0, b)), g["a_f0"]) < TOL
    assert rel(ps.shot_contribution(n(1, b), mask_shot=0.5 * m), g["a_s1"]) < TOL
    assert rel(ps.covariance_contribution(n(2, b), pk_cov, mask_shot=0.5 * m), g["a_c2"]) < TOL
    f, t = ps.theory_contribution(n(3, b), g["kth"], lmax_theory=4)
    assert rel(f, g["a_f3"]) < TOL and rel(t, g["a_t3"]) < TOL
    ps2 = O.OraclePSpec(b, g["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)), applySinv=si, applySinv_transpose=st)
    assert rel(ps2.numerator(synthetic.lognormal(N, L, seed=21).astype(np.float64) * 0.7, "Sinv"), g["b_num"]) < TOL
    assert rel(ps2.fisher_contribution(n(4, b)), g["b_f4"]) < TOL
    assert rel(ps2.covariance_contribution(n(5, b), pk_cov[:2]), g["b_c5"]) < TOL
    lb = O.OracleBase([L] * 3, [N] * 3, boxcenter=g["center"], sightline="local")
    lsi, lst = sinv_pair(lb, N)
    lps = O.OraclePSpec(lb, g["edges"], lmax=2, mask=m, applySinv=lsi, applySinv_transpose=lst)
    assert rel(lps.numerator(d, "Sinv"), g["c_num"]) < TOL
    assert rel(lps.fisher_contribution(n(6, lb)), g["c_f6"]) < TOL
    assert rel(lps.shot_contribution(n(7, lb), mask_shot=0.5 * m), g["c_s7"]) < TOL
    ps4 = O.OraclePSpec(b, g["edges"], lmax=2, mask=m, applySinv=si)
    assert rel(ps4.fisher_contribution(n(8, b)), g["d_f8"]) < TOL


def test_bk_custom_sinv():
    """BSpec with a caller's S^-1: numerator with and without the linear term, Fisher, shot
    noise, covariance; and a constant mask."""
    g = gold("bk_custom_sinv")
    N, L = int(g["N"]), float(g["L"])
    m = mask24(N, L)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * m
    b = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic")
    si, st = sinv_pair(b, N)
    bs = O.OracleBSpec(b, g["edges"], lmax=2, mask=m, applySinv=si, applySinv_transpose=st)
    assert np.array_equal(bs.all_bins, g["bins"])
    sym = g["sym"]
    cub = bs.numerator(d, "Sinv", sym=sym)
    assert rel(cub, g["cub"]) < TOL
    sims = [bs.generated_sim(i) for i in range(2)]
    num = bs.numerator(d, "Sinv", sym=sym, sims=sims)
    assert rel(num, g["num"]) < TOL and rel(num - cub, g["num"] - g["cub"]) < 1e-8
    n = lambda s: (b.reference_noise(s + 10 ** 7), b.reference_noise(s + 2 * 10 ** 7))
    assert rel(bs.fisher_contribution(*n(0), sym=sym), g["f0"]) < TOL
    assert rel(bs.shot_contribution(*n(1), 0.5 * m, data=d, data2=0.7 * d, sym=sym), g["s1"]) < TOL
    pk_cov = [g["pk_k"], g["p0"], g["p2"]]
    assert rel(bs.covariance_contribution(*n(2), pk_cov, mask_shot_2pt=0.5 * m, sym=sym), g["c2"]) < TOL
    bs2 = O.OracleBSpec(b, g["edges"], lmax=2, mask=0.7 * np.ones((N, N, N)), applySinv=si, applySinv_transpose=st)
    d2 = synthetic.lognormal(N, L, seed=21).astype(np.float64) * 0.7
    assert rel(bs2.numerator(d2, "Sinv", sym=sym), g["b_cub"]) < TOL
    assert rel(bs2.fisher_contribution(*n(3), sym=sym), g["b_f3"]) < TOL
