"""Parity at the headline size through size-independent properties: the 256^3 box of side
2000 Mpc/h with the TSC window, 16 linear bins from 2 pi/2000 to 0.2 h/Mpc, lmax = 2, on the
seeded lognormal field the benchmark uses.

* Homogeneity: the numerators are quadratic (Pk) and cubic (Bk) in the data, and doubling a
  field scales every FP64 operation exactly, so num(2 d) = 4 num(d) and 8 num(d) up to the
  order of the atomic accumulations (1e-12 relative).
* Precision modes: the mixed-precision path (FP32 transforms and maps, the CUDA-core or the
  tensor-core contraction -- the latter through both cubic-sum routes -- FP64 sums) against
  the FP64 path on the same field, 1e-5 of each multipole block's largest |value| (the
  mixed-precision bound)."""
import contextlib
import io

import numpy as np
import pytest

from polybin3d_b200 import synthetic

pytestmark = pytest.mark.gpu
N, L = 256, 2000.0
EDGES = np.linspace(2 * np.pi / L, 0.2, 17)


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def blocks(a, b, n_blocks):
    nb = len(b) // n_blocks
    return max(rel(a[j * nb:(j + 1) * nb], b[j * nb:(j + 1) * nb]) for j in range(n_blocks))


@pytest.fixture(scope="module")
def field():
    return synthetic.lognormal(N, L, seed=0)


@pytest.fixture(scope="module")
def bases():
    import polybin3d_b200 as pb
    return {p: quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda", precision=p)
            for p in ("fp64", "mixed")}


def test_pk_headline(bases, field):
    import polybin3d_b200 as pb
    d = field.astype(np.float64)
    ps = quiet(pb.PSpec, bases["fp64"], EDGES, lmax=2)
    ref = ps.Pk_numerator_ideal(d)
    assert rel(ps.Pk_numerator_ideal(2.0 * d), 4.0 * ref) < 1e-12
    psm = quiet(pb.PSpec, bases["mixed"], EDGES, lmax=2)
    assert blocks(psm.Pk_numerator_ideal(field), ref, 2) < 1e-5


@pytest.fixture(scope="module")
def bk_ref(bases, field):
    """The FP64 numerator (and its doubled-field check)."""
    import polybin3d_b200 as pb
    d = field.astype(np.float64)
    bs = quiet(pb.BSpec, bases["fp64"], EDGES, lmax=2)
    ref = quiet(bs.Bk_numerator_ideal, d)
    assert rel(quiet(bs.Bk_numerator_ideal, 2.0 * d), 8.0 * ref) < 1e-12
    return bs.all_bins, ref


def test_bk_headline(bases, field, bk_ref):
    import polybin3d_b200 as pb
    bins, ref = bk_ref
    bsm = quiet(pb.BSpec, bases["mixed"], EDGES, lmax=2, contraction="simt")
    assert np.array_equal(bsm.all_bins, bins)
    assert blocks(quiet(bsm.Bk_numerator_ideal, field), ref, 2) < 1e-5


def test_bk_headline_tensor_cores(bases, field, bk_ref):
    """The benchmark's contraction: tensor cores, through the public call (the route the
    autotuner picks) and through each cubic-sum route (tiled set, plain maps) on its own."""
    import torch
    import polybin3d_b200 as pb
    from polybin3d_b200.bspec import tc_available
    if not tc_available():
        pytest.skip("tensor-core contraction needs sm_100")
    bins, ref = bk_ref
    b = bases["mixed"]
    bsm = quiet(pb.BSpec, b, EDGES, lmax=2, contraction="tc")
    assert np.array_equal(bsm.all_bins, bins)
    assert blocks(quiet(bsm.Bk_numerator_ideal, field), ref, 2) < 1e-5
    norm = b.volume / float(b.gridsize.prod()) / bsm.sym_factor
    xk = bsm._data_spectrum(b.as_device(field))
    w = bsm._data_weight(torch.float32)
    scale = 1.0 / bsm.cube_mask_mean ** (1. / 3.)
    for route in (bsm._b3_tiled, bsm._b3_plain):
        assert blocks(route(xk, w, scale).cpu().numpy() * norm, ref, 2) < 1e-5, route.__name__
