"""Host-side pieces of the Monte Carlo matrices that run as torch code on any device, checked
on CPU tensors against the oracle (itself pinned to the reference's outputs): the pointing
matrix with the global and radial integral constraints (and its transpose), the real
spherical harmonics l = 1..4, and the wide-angle derivative coefficients."""
import types

import numpy as np
import torch

from oracle import polybin_oracle as O
from polybin3d_b200 import pointing
from polybin3d_b200.harmonics import real_harmonics
from polybin3d_b200.pspec import PSpec


def _box(N=12, L=600.0, center=(700.0, 400.0, 900.0)):
    r_arrs = [np.fft.fftshift(np.arange(-N // 2, N // 2)) * L / N + center[i] for i in range(3)]
    r_grids = np.meshgrid(*r_arrs, indexing="ij")
    base = types.SimpleNamespace(device=torch.device("cpu"), nreal=N ** 3, r_grids=r_grids)
    return base, r_grids


def _maps(N, n, seed):
    rng = np.random.default_rng(seed)
    mask = rng.uniform(0.0, 1.0, (N, N, N)) * (rng.uniform(size=(N, N, N)) > 0.3)
    return mask, (mask > 0).astype(np.float64), rng.standard_normal((n, N, N, N))


def test_pointing_global_constraint():
    N = 12
    base, _ = _box(N)
    mask, mic, x = _maps(N, 3, 0)
    P = pointing.Pointing(base, torch.as_tensor(mask), mic, "GIC")
    ref = O.Pointing(mask, mic, "GIC")
    xt = torch.as_tensor(x)
    for tr in (False, True):
        got = P(xt, tr).numpy()
        want = np.stack([ref(x[i], tr) for i in range(3)])
        assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))
    out = xt.clone()
    P(out, True, out=out)
    assert np.max(np.abs(out.numpy() - np.stack([ref(x[i], True) for i in range(3)]))) < 1e-12


def test_pointing_radial_constraint():
    N = 12
    base, r_grids = _box(N)
    mask, mic, x = _maps(N, 2, 1)
    edges = np.array([1000.0, 1150.0, 1250.0, 1350.0, 1500.0])
    modr = np.sqrt(r_grids[0] ** 2 + r_grids[1] ** 2 + r_grids[2] ** 2)
    P = pointing.Pointing(base, torch.as_tensor(mask), mic, "RIC", edges)
    ref = O.Pointing(mask, mic, "RIC", edges, modr)
    assert ((modr < edges[0]) | (modr >= edges[-1])).any(), "some voxels lie outside every shell"
    for tr in (False, True):
        got = P(torch.as_tensor(x), tr).numpy()
        want = np.stack([ref(x[i], tr) for i in range(2)])
        assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))
        outside = (modr < edges[0]) | (modr >= edges[-1])
        assert np.all(got[:, outside] == 0.0)


def test_real_harmonics_all_l():
    rng = np.random.default_rng(3)
    grids = list(rng.standard_normal((3, 5, 6, 7)))
    grids[0][0, 0, 0] = grids[1][0, 0, 0] = grids[2][0, 0, 0] = 0.0
    want = O.real_harmonics_fourier(grids, 4)
    for l in (1, 2, 3, 4):
        got = np.asarray(real_harmonics(grids, l))
        assert got.shape[0] == 2 * l + 1
        assert np.max(np.abs(got - want[l])) < 1e-14
    # addition theorem with the reference's normalisation: sum_m Y_lm(n) Y_lm(n) = L_l(1) = 1
    n = np.asarray(grids)[:, 1:, 1:, 1:]
    for l in (1, 2, 3, 4):
        y = np.asarray(real_harmonics(list(n), l))
        assert np.allclose((y * y).sum(0), 1.0, atol=1e-12)


def test_wide_angle_derivative_coefficients():
    for k in (np.linspace(0.01, 0.12, 7), np.geomspace(0.01, 0.2, 5)):
        assert np.array_equal(PSpec.derivative_coefficient(k), O.OraclePSpec.derivative_coefficient(k))


def test_route_chooser_cache_and_disabled(tmp_path, monkeypatch):
    """autotune.Tuner.choose_route: a cached winner is returned without running anything; with
    tuning off the first route is taken, also without running anything."""
    import json
    from polybin3d_b200 import autotune

    def never():
        raise AssertionError("a route ran")

    path = tmp_path / "tuning.json"
    path.write_text(json.dumps({"b3route|dev|192,192,192|32|16|global": {"route": "plain"}}))
    monkeypatch.setenv("PB_TUNING_CACHE", str(path))
    t = autotune.Tuner()
    assert t.choose_route("b3route|dev|192,192,192|32|16|global", {"tiled": never, "plain": never}) == "plain"
    monkeypatch.setenv("PB_AUTOTUNE", "0")
    assert t.choose_route("another|key", {"tiled": never, "plain": never}) == "tiled"
    assert "another|key" not in json.loads(path.read_text())
