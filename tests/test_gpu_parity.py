"""Parity of the CUDA path (public API -> C ABI -> sm_100a kernels) with the reference.

Fixtures under tests/golden/ were produced by the reference itself; the oracle
(oracle/polybin_oracle.py) checks cases without a fixture on the same seeded inputs.
Tolerances: FP64 mode 1e-10 relative (Fisher MC 1e-8), mixed mode 1e-5 relative with the
per-bin floor 1e-3 * max|ref| of the block."""
import contextlib
import io
import os

import numpy as np
import pytest
import torch

from polybin3d_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


def rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def rel_floor(a, b, floor=1e-3):
    """max_i |a_i - b_i| / max(|b_i|, floor * max|b|)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(b), floor * np.max(np.abs(b)))
    return np.max(np.abs(a - b) / den)


def mixed_err(a, b):
    """Mixed-precision metric: max_i |a_i - b_i| / max_i |b_i| over one multipole block.
    FP32 transforms put an absolute error of ~1e-6 of the block's largest |B| on every
    bin, so bins that cross zero (quadrupoles) cannot meet a per-bin relative bound."""
    return rel(a, b)


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def field(g):
    kind, seed, N, L = str(g["data_kind"]), int(g["data_seed"]), int(g["N"]), float(g["L"])
    return synthetic.grf(N, L, seed) if kind == "grf" else synthetic.lognormal(N, L, seed)


def mask24(N, L):
    return synthetic.shell_mask(N, L, r_in=L / 6, r_out=0.4667 * L, n_holes=10, hole_r=(10.0, 30.0),
                                hole_box=0.4667 * L, seed=0)


@pytest.fixture(scope="module")
def pb():
    import polybin3d_b200
    return polybin3d_b200


def base(pb, g, pw="none", precision="fp64", Pk=None):
    N, L = int(g["N"]), float(g["L"])
    return quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=Pk, pixel_window=pw, backend="cuda", precision=precision)


def test_mode_counts_bit_exact(pb):
    """Mode counts per bin (integrate of ones) equal the oracle's exactly."""
    from oracle import polybin_oracle as O
    for N, L, edges in [(64, 1000.0, None), (32, 500.0, np.linspace(2 * np.pi / 500, 0.2, 9))]:
        kF = 2 * np.pi / L
        e = kF + 2 * kF * np.arange(11) if edges is None else edges
        b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, backend="cuda")
        ps = quiet(pb.PSpec, b, e, lmax=0)
        out = torch.empty(ps.Nk, dtype=torch.float64, device=b.device)
        from polybin3d_b200 import _native as nat
        nat.bin_reduce(b.grid, nat.PB_F64, nat.PB_RED_REAL2, None, None, 1, e, [(0, 0)], 1.0, out, b.ws)
        ob = O.OracleBase([L] * 3, [N] * 3)
        ref = ob.real_integrate_double(np.ones(ob.modk_grid.shape), 0, 0, e)
        assert np.array_equal(out.cpu().numpy(), ref)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_cfg1_pk_ideal(pb, precision, tol):
    g = gold("cfg1")
    b = base(pb, g, precision=precision)
    ps = quiet(pb.PSpec, b, g["edges"], lmax=2)
    d = field(g)
    assert rel(quiet(ps.Pk_numerator_ideal, d), g["pk_num"]) < tol
    pk = quiet(ps.Pk_ideal, d)
    assert rel(ps.fish_ideal, g["pk_fish"]) < 1e-12
    for k in pk:
        assert (rel if precision == "fp64" else mixed_err)(pk[k], g["Pk_" + k]) < tol


@pytest.mark.parametrize("precision,contraction,tol", [("fp64", "simt", 1e-10), ("mixed", "simt", 1e-5),
                                                       ("mixed", "auto", 1e-5)])
def test_cfg1_bk_ideal(pb, precision, contraction, tol):
    g = gold("cfg1")
    b = base(pb, g, precision=precision)
    bs = quiet(pb.BSpec, b, g["edges"], lmax=0, contraction=contraction)
    assert np.array_equal(bs.all_bins, g["bk_bins"])
    d = field(g)
    bk = quiet(bs.Bk_ideal, d)
    assert np.array_equal(bs.sym_factor, g["bk_sym"])
    assert rel(bs.fish_ideal, g["bk_fish"]) < 1e-10
    err = rel if precision == "fp64" else mixed_err
    assert err(quiet(bs.Bk_numerator_ideal, d), g["bk_num"]) < tol
    assert err(bk["b0"], g["Bk_b0"]) < tol


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_bk_lmax2_tsc(pb, precision, tol):
    g = gold("bk_l2_tsc")
    b = base(pb, g, pw="tsc", precision=precision)
    bs = quiet(pb.BSpec, b, g["edges"], lmax=2)
    d = field(g)
    bk = quiet(bs.Bk_ideal, d)
    assert rel(bs.sym_factor, g["bk_sym"]) < 1e-10
    assert rel(bs.fish_ideal, g["bk_fish"]) < 1e-10
    num = quiet(bs.Bk_numerator_ideal, d)
    n3 = bs.N3
    err = rel if precision == "fp64" else mixed_err
    for blk in range(bs.Nl):
        sl = slice(blk * n3, (blk + 1) * n3)
        assert err(num[sl], g["bk_num"][sl]) < tol
    for k in bk:
        assert err(bk[k], g["Bk_" + k]) < tol
    bs2 = quiet(pb.BSpec, b, g["edges"], lmax=2)
    assert rel(quiet(bs2.compute_fisher_ideal, discreteness_correction=False), g["bk_fish_nodisc"]) < 1e-10


def test_bk_squeezed_partial(pb):
    g = gold("bk_squeeze_partial")
    b = base(pb, g, pw="cic")
    bs = quiet(pb.BSpec, b, g["edges"], lmax=0, k_bins_squeeze=g["edges_sq"], include_partial_triangles=True)
    assert np.array_equal(bs.all_bins, g["bk_bins"])
    bk = quiet(bs.Bk_ideal, field(g))
    assert rel(bk["b0"], g["Bk_b0"]) < 1e-10


@pytest.mark.parametrize("pw", ["cic", "interlaced-tsc"])
def test_pk_windows(pb, pw):
    g = gold("pk_windows")
    b = base(pb, g, pw=pw, Pk=synthetic.pk_table(1.0))
    ps = quiet(pb.PSpec, b, g["edges"], lmax=4)
    tag = pw.replace("-", "_")
    d = field(g)
    assert rel(quiet(ps.Pk_numerator_ideal, d), g[tag + "_num"]) < 1e-10
    assert rel(quiet(ps.compute_fisher_ideal), g[tag + "_fish"]) < 1e-10
    pk = quiet(ps.Pk_ideal, d)
    for k in pk:
        assert rel(pk[k], g[tag + "_Pk_" + k]) < 1e-10
    ps2 = quiet(pb.PSpec, b, g["edges"], lmax=4)
    assert rel(quiet(ps2.compute_fisher_ideal, discreteness_correction=False), g[tag + "_fish_nodisc"]) < 1e-10


def test_generate_data_matches_reference(pb):
    g = gold("grf_noise")
    b = base(pb, g, pw="cic", Pk=synthetic.pk_table(1.0))
    a = b.generate_data(seed=int(g["seed"]), output_type="fourier").cpu().numpy()
    assert np.max(np.abs(a - g["a"])) / np.max(np.abs(g["a"])) < 1e-14


def test_pk_fisher_masked(pb):
    g = gold("pk_fisher_mask")
    N, L = int(g["N"]), float(g["L"])
    b = base(pb, g)
    ps = quiet(pb.PSpec, b, g["edges"], lmax=4, mask=mask24(N, L))
    f0 = quiet(ps.compute_fisher_contribution, 0)
    assert rel(f0, g["f0"]) < 1e-10
    fish = quiet(ps.compute_fisher, 2)
    assert rel(fish, 0.5 * (g["f0"] + g["f1"])) < 1e-10
    data = synthetic.lognormal(N, L, seed=int(g["data_seed"])).astype(np.float64) * mask24(N, L)
    pk = quiet(ps.Pk_unwindowed, data)
    for k in pk:
        assert rel(pk[k], g["Pk_" + k]) < 1e-8


def test_pk_fisher_nomask(pb):
    g = gold("pk_fisher_nomask")
    b = base(pb, g, pw="tsc")
    ps = quiet(pb.PSpec, b, g["edges"], lmax=2)
    assert rel(quiet(ps.compute_fisher_contribution, 2), g["f2"]) < 1e-10


def test_bk_fisher_masked(pb):
    g = gold("bk_fisher_mask")
    N, L = int(g["N"]), float(g["L"])
    b = base(pb, g)
    m = mask24(N, L)
    bs = quiet(pb.BSpec, b, g["edges"], lmax=0, mask=m)
    assert np.array_equal(bs.all_bins, g["bins0"])
    f0 = quiet(bs.compute_fisher_contribution, 0)
    assert rel(f0, g["f0"]) < 1e-8
    data = synthetic.lognormal(N, L, seed=int(g["data_seed"])).astype(np.float64) * m
    num = quiet(bs.Bk_numerator, data, include_linear_term=False)
    assert rel(num, g["num0"]) < 1e-10
    bk = quiet(bs.Bk_unwindowed, data, fish=g["f0"], include_linear_term=False)
    assert rel(bk["b0"], g["Bk_b0"]) < 1e-8
    bs2 = quiet(pb.BSpec, b, g["edges"], lmax=2, mask=m)
    assert rel(quiet(bs2.compute_fisher_contribution, 0), g["f2_l2"]) < 1e-8


def test_bk_fisher_nomask_lmax2(pb):
    g = gold("bk_fisher_nomask")
    b = base(pb, g, pw="cic")
    bs = quiet(pb.BSpec, b, g["edges"], lmax=2)
    assert rel(quiet(bs.compute_fisher_contribution, 3), g["f3"]) < 1e-8


def test_unwindowed_needs_fisher_and_sims(pb):
    g = gold("bk_fisher_nomask")
    b = base(pb, g)
    bs = quiet(pb.BSpec, b, g["edges"], lmax=0)
    with pytest.raises(Exception, match="Need to compute Fisher matrix first!"):
        bs.Bk_unwindowed(synthetic.grf(int(g["N"]), float(g["L"]), 0))
    with pytest.raises(Exception, match="Need to generate or specify bias simulations!"):
        bs.Bk_unwindowed(synthetic.grf(int(g["N"]), float(g["L"]), 0), fish=np.eye(bs.N_bins))
    ps = quiet(pb.PSpec, b, g["edges"], lmax=0)
    with pytest.raises(Exception, match="Need to compute Fisher matrix first!"):
        ps.Pk_unwindowed(synthetic.grf(int(g["N"]), float(g["L"]), 0))


def test_dealiased_map_grid_is_exact(pb):
    """Maps synthesised on the coarse grid M > 3K give the same bispectrum as full-grid maps."""
    from oracle import polybin_oracle as O
    N, L = 64, 1000.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.06, 5)
    d = synthetic.lognormal(N, L, seed=5)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="cuda")
    bs = quiet(pb.BSpec, b, edges, lmax=2)
    assert bs.map_grid[0] < N
    bs_full = quiet(pb.BSpec, b, edges, lmax=2, dealias=False)
    assert bs_full.map_grid == (N, N, N)
    r1 = quiet(bs.Bk_ideal, d)
    r2 = quiet(bs_full.Bk_ideal, d)
    ob = O.OracleBase([L] * 3, [N] * 3, pixel_window="cic")
    ref = O.OracleBSpec(ob, edges, lmax=2).Bk_ideal(d)
    for k in ref:
        assert rel(r1[k], ref[k]) < 1e-10
        assert rel(r2[k], ref[k]) < 1e-10
    assert rel(bs.sym_factor, bs_full.sym_factor) < 1e-10


def test_bk_ideal_streamed_list(pb):
    """Bk_ideal on a list of fields (copies overlapped on a side stream) equals field-by-field."""
    N, L = 48, 600.0
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision="mixed")
    bs = quiet(pb.BSpec, b, np.linspace(2 * np.pi / L, 0.11, 6), lmax=2)
    fields = [torch.from_numpy(synthetic.lognormal(N, L, seed=s)).pin_memory() for s in range(3)]
    fields.append(synthetic.lognormal(N, L, seed=7))  # a numpy field in the same list
    one = [quiet(bs.Bk_ideal, f if isinstance(f, np.ndarray) else f.numpy()) for f in fields]
    many = quiet(bs.Bk_ideal, fields)
    assert len(many) == len(fields)
    for a, r in zip(many, one):
        for k in r:
            assert rel(a[k], r[k]) < 1e-12
