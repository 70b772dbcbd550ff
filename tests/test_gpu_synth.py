"""pb_shell_synth (band-limited filter + inverse real transform in one pruned pass) against
the two-step form it replaces: pb_spectral_filter onto the output grid, then the cuFFT C2R.
Non-cubic grids and boxes, a smaller output grid, two sources, Legendre weights, window
powers and more than one chunk of maps; FP64 and FP32."""
import contextlib
import io

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def quiet(fn, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


@pytest.fixture(scope="module")
def pb():
    import polybin3d_b200
    return polybin3d_b200


CASES = [
    # data grid, box, output grid (None = same)
    ((24, 24, 24), (600.0, 600.0, 600.0), None),
    ((48, 48, 48), (600.0, 600.0, 600.0), (32, 32, 32)),
    ((32, 40, 48), (700.0, 500.0, 900.0), None),
    ((64, 64, 64), (1000.0, 1000.0, 1000.0), (30, 30, 30)),
]


def maps_for(b, outn, n_maps, rng):
    kny = min(np.pi * outn[i] / b.boxsize[i] for i in range(3))
    top = 0.9 * kny
    edges = np.linspace(np.max(b.kF), top, 9)
    out = []
    for m in range(n_maps):
        i = m % 8
        out.append((m % 2, edges[i], edges[i + 1], [0, 2, 4][m % 3], [0, 2][(m // 3) % 2], float(rng.uniform(0.5, 2)),
                    [0, 1, -1, 2][m % 4]))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_shell_synth_matches_filter_then_c2r(pb, precision, case):
    from polybin3d_b200 import _native as nat
    N, L, outn = CASES[case]
    outn = outn or N
    b = quiet(pb.PolyBin3D, list(L), list(N), pixel_window="cic", backend="cuda", precision=precision)
    rd = torch.float64 if precision == "fp64" else torch.float32
    prec = nat.precision_of(rd)
    g = torch.Generator().manual_seed(case)
    x = torch.randn((2,) + tuple(N), generator=g, dtype=torch.float64).to(rd).to(b.device)
    src = b.fft_r2c(x)
    w = b.to_device_grid("window", lambda: b.pixel_window_grid, rd)
    rng = np.random.default_rng(case)
    n_maps = 70 if case == 0 else 12
    maps = maps_for(b, outn, n_maps, rng)
    hs = (outn[0], outn[1], outn[2] // 2 + 1)
    half = torch.empty((n_maps,) + hs, dtype=src.dtype, device=b.device)
    nat.spectral_filter(b.grid, prec, src, half, maps, w=w, out_n=list(outn))
    ref = b.fft_c2r(half).cpu().numpy()
    out = torch.empty((n_maps,) + tuple(outn), dtype=rd, device=b.device)
    nat.shell_synth(b.grid, prec, src, out, maps, list(outn), b.ws, w=w)
    out = out.cpu().numpy()
    tol = 1e-12 if precision == "fp64" else 5e-6
    for m in range(n_maps):
        scale = np.max(np.abs(ref[m]))
        assert scale > 0
        assert np.max(np.abs(out[m] - ref[m])) / scale < tol, (m, maps[m])


def test_shell_synth_refuses_unbounded_bands(pb):
    from polybin3d_b200 import _native as nat
    b = quiet(pb.PolyBin3D, [600.0] * 3, [24] * 3, backend="cuda")
    src = b.fft_r2c(torch.randn((24,) * 3, dtype=torch.float64, device=b.device))
    out = torch.empty((1, 24, 24, 24), dtype=torch.float64, device=b.device)
    with pytest.raises(NotImplementedError):
        nat.shell_synth(b.grid, nat.PB_F64, src, out, [(0, 0.0, np.inf, 0, 0, 1.0, 0)], [24] * 3, b.ws)
    with pytest.raises(NotImplementedError):   # reaches the Nyquist frequency of the grid
        nat.shell_synth(b.grid, nat.PB_F64, src, out, [(0, 0.0, 0.99 * np.pi * 24 / 600.0, 0, 0, 1.0, 0)],
                        [24] * 3, b.ws)


def test_bk_numerator_pruned_equals_cufft(pb):
    """The bispectrum numerator through both synthesis paths (dealiased map grid)."""
    from polybin3d_b200 import synthetic
    N, L = 48, 600.0
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="cuda")
    edges = np.linspace(2 * np.pi / L, 0.11, 6)
    d = synthetic.lognormal(N, L, seed=2).astype(np.float64)
    r = {}
    for mode in ("pruned", "cufft"):
        bs = quiet(pb.BSpec, b, edges, lmax=2, synthesis=mode)
        r[mode] = quiet(bs.Bk_numerator_ideal, d)
    assert np.max(np.abs(r["pruned"] - r["cufft"])) / np.max(np.abs(r["cufft"])) < 1e-12


@pytest.mark.parametrize("case", [1, 2])
def test_shell_synth_f32_maps_from_f64_source(pb, case):
    """PB_F32_SRC_F64: FP32 maps (FP32 weights) read straight from a complex128 spectrum,
    against the FP64 synthesis of the same spectrum (one FP32 rounding of the filtered modes
    and FP32 transforms: 2e-6 of each map's largest value), and as a tiled set, whose factor
    rows must equal the plain maps exactly."""
    from polybin3d_b200 import _native as nat
    N, L, outn = CASES[case]
    outn = outn or N
    b = quiet(pb.PolyBin3D, list(L), list(N), pixel_window="cic", backend="cuda")
    g = torch.Generator().manual_seed(10 + case)
    x = torch.randn((2,) + tuple(N), generator=g, dtype=torch.float64).to(b.device)
    src = b.fft_r2c(x)
    w64 = b.to_device_grid("window", lambda: b.pixel_window_grid, torch.float64)
    w32 = w64.float()
    maps = maps_for(b, outn, 12, np.random.default_rng(case))
    ref = torch.empty((12,) + tuple(outn), dtype=torch.float64, device=b.device)
    nat.shell_synth(b.grid, nat.PB_F64, src, ref, maps, list(outn), b.ws, w=w64)
    out = torch.empty((12,) + tuple(outn), dtype=torch.float32, device=b.device)
    nat.shell_synth(b.grid, nat.PB_F32_SRC_F64, src, out, maps, list(outn), b.ws, w=w32)
    ref, o = ref.cpu().numpy(), out.cpu().numpy()
    for m in range(12):
        scale = np.max(np.abs(ref[m]))
        assert np.max(np.abs(o[m] - ref[m])) / scale < 2e-6, (m, maps[m])
    T = nat.TiledMaps(12, 4, tuple(outn), b.device)
    nat.shell_synth(b.grid, nat.PB_F32_SRC_F64, src, T, maps, list(outn), b.ws, w=w32)
    assert torch.equal(T.factor_maps().reshape(4, -1), out[:4].reshape(4, -1))


@pytest.mark.parametrize("n", [1, 3, 4, 1001, 64 ** 3 + 2])
def test_widen_exact(n):
    """PB_EW_WIDEN: the FP32 -> FP64 copy before the data's FP64 transform, exact for every
    length (vectorised body and scalar tail) and for an unaligned start."""
    from polybin3d_b200 import _native as nat
    x = torch.randn(n + 1, generator=torch.Generator().manual_seed(n)).to("cuda")
    assert torch.equal(nat.widen(x[:n].contiguous()), x[:n].double())
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    nat.check(nat.load().pb_elementwise(nat.PB_F32, nat.PB_EW_WIDEN, n, nat.ctypes.c_void_p(x.data_ptr() + 4), None, 0,
                                        None, None, 0.0, nat.ptr(y), nat.stream_ptr()), "pb_elementwise")
    assert torch.equal(y, x[1:].double())
