"""Parity at the headline size through size-independent properties: the 256^3 box of side
2000 Mpc/h with the TSC window, 16 linear bins from 2 pi/2000 to 0.2 h/Mpc, lmax = 2, on the
seeded lognormal field the benchmark uses.

* Homogeneity: the numerators are quadratic (Pk) and cubic (Bk) in the data, and doubling a
  field scales every FP64 operation exactly, so num(2 d) = 4 num(d) and 8 num(d) up to the
  order of the atomic accumulations (1e-12 relative).
* Precision modes: the mixed-precision path (FP32 transforms and maps, CUDA-core FP32
  contraction, FP64 sums) against the FP64 path on the same field, 1e-5 of each multipole
  block's largest |value| (the mixed-precision bound)."""
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


def test_bk_headline(bases, field):
    import polybin3d_b200 as pb
    d = field.astype(np.float64)
    bs = quiet(pb.BSpec, bases["fp64"], EDGES, lmax=2)
    ref = quiet(bs.Bk_numerator_ideal, d)
    assert rel(quiet(bs.Bk_numerator_ideal, 2.0 * d), 8.0 * ref) < 1e-12
    bsm = quiet(pb.BSpec, bases["mixed"], EDGES, lmax=2, contraction="simt")
    assert np.array_equal(bsm.all_bins, bs.all_bins)
    assert blocks(quiet(bsm.Bk_numerator_ideal, field), ref, 2) < 1e-5
