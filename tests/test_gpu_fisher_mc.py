"""Monte Carlo Fisher in throughput mode: white noise drawn on the device (Philox4x32-10
keyed by the seed) and each batch of realisations replayed from one captured CUDA graph.
Checked against the oracle fed the same Philox noise (restated in numpy and pinned to the
generator's known-answer vectors), and against the uncaptured device path."""
import contextlib
import io

import numpy as np
import pytest

from polybin3d_b200 import synthetic

pytestmark = pytest.mark.gpu


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def mask24(N, L):
    return synthetic.shell_mask(N, L, r_in=L / 6, r_out=0.4667 * L, n_holes=10, hole_r=(10.0, 30.0),
                                hole_box=0.4667 * L, seed=0)


@pytest.fixture(scope="module")
def pb():
    import polybin3d_b200
    return polybin3d_b200


@pytest.mark.parametrize("pw", ["none", "cic"])
def test_grf_philox_matches_oracle(pb, pw):
    from oracle import polybin_oracle as O
    N, L = 24, 600.0
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window=pw, backend="cuda")
    ob = O.OracleBase([L] * 3, [N] * 3, pixel_window=pw)
    a = b.grf_philox([7, 2 ** 40 + 3]).cpu().numpy()
    for i, s in enumerate([7, 2 ** 40 + 3]):
        ref = ob.grf_from_noise(*ob.philox_noise(s))
        assert rel(a[i], ref) < 1e-13


def test_pk_fisher_philox_graph(pb):
    from oracle import polybin_oracle as O
    N, L = 24, 600.0
    edges = np.linspace(2 * np.pi / L, 0.11, 5)
    m = mask24(N, L)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, backend="cuda")
    ps = quiet(pb.PSpec, b, edges, lmax=4, mask=m)
    n_it = 5  # batches of 2: two full replays and one padded replay
    fish = quiet(ps.compute_fisher, n_it, batch=2, noise="philox")
    # the uncaptured device path on the same seeds
    eager = ps._fisher_from_fields(b.grf_philox([s + int(1e7) for s in range(n_it)])).cpu().numpy()
    assert rel(fish, eager.mean(axis=0)) < 1e-14
    # the oracle on the same noise
    ob = O.OracleBase([L] * 3, [N] * 3)
    ops = O.OraclePSpec(ob, edges, lmax=4, mask=m)
    ref = np.mean([ops.fisher_contribution(ob.philox_noise(s + int(1e7))) for s in range(n_it)], axis=0)
    assert rel(fish, ref) < 1e-10
    # a second call replays the same graph (the k-bin reductions accumulate with shared-memory
    # atomics, so repeated runs agree to rounding, not bit for bit)
    assert rel(quiet(ps.compute_fisher, n_it, batch=2, noise="philox"), fish) < 1e-14


def test_bk_fisher_philox_graph(pb):
    from oracle import polybin_oracle as O
    N, L = 24, 600.0
    edges = np.linspace(2 * np.pi / L, 0.11, 5)
    m = mask24(N, L)
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, backend="cuda")
    bs = quiet(pb.BSpec, b, edges, lmax=0, mask=m)
    fish = quiet(bs.compute_fisher, 2, noise="philox")
    eager = [bs._fisher_from_fields(b.grf_philox([s + int(1e7)]), b.grf_philox([s + int(2e7)])).cpu().numpy()
             for s in range(2)]
    assert rel(fish, 0.5 * (eager[0] + eager[1])) < 1e-14
    ob = O.OracleBase([L] * 3, [N] * 3)
    obs = O.OracleBSpec(ob, edges, lmax=0, mask=m)
    sym = obs.symmetry_factor()
    ref = np.mean([obs.fisher_contribution(ob.philox_noise(s + int(1e7)), ob.philox_noise(s + int(2e7)), sym=sym)
                   for s in range(2)], axis=0)
    assert rel(fish, ref) < 1e-8


def test_fisher_reference_noise_unchanged_by_sharding_code(pb):
    """compute_fisher with the reference noise still reproduces the golden mean (the
    one-process path of the seed-sharding helper)."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pk_fisher_mask.npz"))
    N, L = int(g["N"]), float(g["L"])
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, backend="cuda")
    ps = quiet(pb.PSpec, b, g["edges"], lmax=4, mask=mask24(N, L))
    fish = quiet(ps.compute_fisher, 2, batch=1)
    assert rel(fish, 0.5 * (g["f0"] + g["f1"])) < 1e-10
