"""Q-maps as gradients: the backward kernels of the differentiable numerators
(polybin3d_b200.autograd) against central finite differences of the forward, and
against the reference's own Q-maps captured into the golden fixtures.

Finite differences: the power-spectrum numerator is quadratic in the data, so the central
difference is exact for any step; the bispectrum numerator is cubic, so the step-h and
step-h/2 central differences are combined by one Richardson step, which is again exact.
What remains is rounding, far below the 1e-6 relative bound used here."""
import contextlib
import io
import os

import numpy as np
import pytest
import torch

from polybin3d_b200 import synthetic

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FD_TOL = 1e-6
STEP = 1e-3


def gold(name):
    return np.load(os.path.join(GOLD, name + ".npz"))


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


def make_base(pb, N, L, pw="none"):
    return quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window=pw, backend="cuda")


def directional(fn, d, v, gam, h, cubic):
    """gam . D_v fn(d) by central differences (with one Richardson step when cubic)."""
    def cd(s):
        with torch.no_grad():
            fp = fn(d + s * v)
            fm = fn(d - s * v)
        return float(torch.dot(gam, fp - fm)) / (2 * s)
    if not cubic:
        return cd(h)
    return (4 * cd(0.5 * h) - cd(h)) / 3


def check_fd(fn, d, n_out, cubic, seed=0, n_vox=64):
    """vjp of fn at d against finite differences along a random direction supported on
    n_vox random voxels, and along 4 single voxels."""
    rng = np.random.default_rng(seed)
    dev = d.device
    gam = torch.as_tensor(rng.standard_normal(n_out), device=dev)
    x = d.clone().requires_grad_(True)
    out = fn(x)
    (grad,) = torch.autograd.grad(out, x, grad_outputs=gam)
    h = STEP * float(d.std())
    flat = rng.choice(d.numel(), size=n_vox, replace=False)
    v = torch.zeros_like(d).reshape(-1)
    v[torch.as_tensor(flat, device=dev)] = torch.as_tensor(rng.standard_normal(n_vox), device=dev)
    v = v.reshape(d.shape)
    ad = float(torch.sum(grad * v))
    fd = directional(fn, d, v, gam, h, cubic)
    assert abs(ad - fd) <= FD_TOL * abs(fd), (ad, fd)
    for j in flat[:4]:
        e = torch.zeros_like(d).reshape(-1)
        e[int(j)] = 1.0
        e = e.reshape(d.shape)
        fd = directional(fn, d, e, gam, h, cubic)
        ad = float(grad.reshape(-1)[int(j)])
        assert abs(ad - fd) <= FD_TOL * max(abs(fd), 1e-3 * float(grad.abs().max())), (int(j), ad, fd)
    return grad


# ------------------------------------------------------------------------------------
# power spectrum
# ------------------------------------------------------------------------------------
def test_pk_forward_matches_numerator(pb):
    from polybin3d_b200.autograd import pk_numerator
    N, L = 24, 600.0
    b = make_base(pb, N, L)
    m = mask24(N, L)
    ps = quiet(pb.PSpec, b, np.linspace(2 * np.pi / L, 0.11, 5), lmax=4, mask=m)
    d = synthetic.lognormal(N, L, seed=3).astype(np.float64)
    num = pk_numerator(ps, torch.as_tensor(d, device=b.device)).cpu().numpy()
    assert rel(num, ps.Pk_numerator(d * m)) < 1e-12


@pytest.mark.parametrize("pw,masked", [("none", True), ("tsc", False), ("cic", True)])
def test_pk_gradient_finite_differences(pb, pw, masked):
    from polybin3d_b200.autograd import pk_numerator
    N, L = 24, 600.0
    b = make_base(pb, N, L, pw)
    ps = quiet(pb.PSpec, b, np.linspace(2 * np.pi / L, 0.11, 5), lmax=4, mask=mask24(N, L) if masked else None)
    d = torch.as_tensor(synthetic.lognormal(N, L, seed=4).astype(np.float64), device=b.device)
    grad = check_fd(lambda x: pk_numerator(ps, x), d, ps.N_bins, cubic=False)
    if masked:
        # the data enter only through m * d: no gradient where the mask vanishes
        m = torch.as_tensor(ps.mask, device=b.device)
        assert float(grad[m == 0].abs().max()) == 0.0


def test_pk_q_maps_match_reference(pb):
    """(N^3/V) rfftn(d num_{l b}/d d) at the seed-0 Fisher GRF equals the reference's
    Q_{l b} = rfftn(m irfftn(Theta_b L_l rfftn(m a))) (pspec.py:443-456)."""
    from polybin3d_b200.autograd import q_maps_pk
    g = gold("pk_fisher_mask")
    N, L = int(g["N"]), float(g["L"])
    b = make_base(pb, N, L)
    ps = quiet(pb.PSpec, b, g["edges"], lmax=int(g["pk_lmax"]), mask=mask24(N, L))
    re, im = b.reference_noise(0 + int(1e7))
    a = b.grf_from_noise(torch.as_tensor(re, device=b.device), torch.as_tensor(im, device=b.device))
    q = q_maps_pk(ps, b.to_real(a)).cpu().numpy()
    assert q.shape == g["q0"].shape
    for i in range(q.shape[0]):
        assert rel(q[i], g["q0"][i]) < 1e-10, i


# ------------------------------------------------------------------------------------
# bispectrum
# ------------------------------------------------------------------------------------
def test_bk_forward_matches_numerator(pb):
    from polybin3d_b200.autograd import bk_numerator
    N, L = 24, 600.0
    b = make_base(pb, N, L)
    m = mask24(N, L)
    bs = quiet(pb.BSpec, b, np.linspace(2 * np.pi / L, 0.11, 5), lmax=2, mask=m)
    d = synthetic.lognormal(N, L, seed=5).astype(np.float64)
    num = bk_numerator(bs, torch.as_tensor(d, device=b.device)).cpu().numpy()
    ref = quiet(bs.Bk_numerator, d * m, include_linear_term=False)
    assert rel(num, ref) < 1e-12


@pytest.mark.parametrize("N,pw,masked,lmax", [(24, "none", True, 2), (24, "cic", False, 0), (48, "tsc", False, 2)])
def test_bk_gradient_finite_differences(pb, N, pw, masked, lmax):
    """48^3 with bins to 0.11 puts the maps on a 32^3 dealiased grid: the gradient's
    transforms then run there and are gathered back onto the data grid."""
    from polybin3d_b200.autograd import bk_numerator
    L = 600.0
    b = make_base(pb, N, L, pw)
    bs = quiet(pb.BSpec, b, np.linspace(2 * np.pi / L, 0.11, 5), lmax=lmax, mask=mask24(N, L) if masked else None)
    if N == 48:
        assert tuple(bs.map_grid) != (N, N, N)
    d = torch.as_tensor(synthetic.lognormal(N, L, seed=6).astype(np.float64), device=b.device)
    check_fd(lambda x: bk_numerator(bs, x), d, bs.N_bins, cubic=True)


def test_bk_q_maps_match_reference(pb):
    """Q_Ainv of the reference's bispectrum Fisher (bspec.py:600-664, seed 0, mask applied)
    from gradients: with d_j = irfftn(A^-1 a_j) and no mask,
    sum_legs Theta FT[g1 g1' - g2 g2'] = (N^3 sym_i / V) (rfftn grad_i(d_1) - rfftn grad_i(d_2))."""
    from polybin3d_b200.autograd import bk_numerator
    g = gold("bk_fisher_mask")
    N, L = int(g["N"]), float(g["L"])
    b = make_base(pb, N, L)
    m = mask24(N, L)
    bs = quiet(pb.BSpec, b, g["edges"], lmax=0)
    assert np.array_equal(bs.all_bins, g["bins0"])
    d = []
    for off in (int(1e7), int(2e7)):
        re, im = b.reference_noise(0 + off)
        a = b.grf_from_noise(torch.as_tensor(re, device=b.device), torch.as_tensor(im, device=b.device))
        d.append(b.to_real(b.applyAinv(a, input_type='fourier', output_type='fourier')))
    nb = bs.N_bins
    grads = []
    for dj in d:
        x = dj.clone().requires_grad_(True)
        out = bk_numerator(bs, x)
        rows = []
        for i in range(nb):
            (gi,) = torch.autograd.grad(out[i], x, retain_graph=i + 1 < nb)
            rows.append(np.fft.rfftn(gi.cpu().numpy()))
        grads.append(np.asarray(rows))
    sym = np.asarray(bs.sym_factor)[:, None, None, None]
    q_pre = (N ** 3 * sym / b.volume) * (grads[0] - grads[1])
    q = np.fft.rfftn(m[None] * np.fft.irfftn(q_pre, s=(N, N, N), axes=(1, 2, 3)), axes=(1, 2, 3))
    assert q.shape == g["q0"].shape
    assert rel(q, g["q0"]) < 1e-10


@pytest.mark.parametrize("case", ["even", "odd"])
def test_pk_local_sightline(pb, case):
    """Local sightline: the forward equals the reference's numerator (tests/golden/local_los.npz,
    lmax=4; tests/golden/local_odd.npz, odd_l with lmax=3) and the gradient, which adds the
    adjoint harmonic transform sum_m FT[Y_lm(r) IFT(Y_lm(k) .)], matches finite differences."""
    from polybin3d_b200.autograd import pk_numerator
    if case == "even":
        g = gold("local_los")
        N, L = int(g["N"]), float(g["L"])
        b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=list(g["center"]), sightline="local",
                  pixel_window="cic", backend="cuda")
        ps = quiet(pb.PSpec, b, g["edges"], lmax=4, mask=mask24(N, L))
        want = g["pk_num"]
    else:
        g = gold("local_odd")
        N, L = int(g["N"]), float(g["L"])
        b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=[g["pk_k"], g["pk_p"]], boxcenter=list(g["center"]),
                  sightline="local", pixel_window="tsc", backend="cuda")
        ps = quiet(pb.PSpec, b, g["edges"], lmax=3, mask=mask24(N, L), odd_l=True)
        want = g["num"]
    d = torch.as_tensor(synthetic.lognormal(N, L, seed=21).astype(np.float64), device=b.device)
    num = pk_numerator(ps, d).cpu().numpy()
    nb = ps.Nk
    for j in range(ps.Nl):
        assert rel(num[j * nb:(j + 1) * nb], want[j * nb:(j + 1) * nb]) < 1e-10, j
    # the mask covers a few per cent of the voxels: spread the direction over enough of them
    # that it reaches inside the mask
    check_fd(lambda x: pk_numerator(ps, x), d, ps.N_bins, cubic=False, seed=5, n_vox=4096)


def test_bk_local_sightline(pb):
    """Local sightline, lmax=2: the forward equals the reference's numerator without the linear
    term (tests/golden/local_los.npz) and the gradient, whose l = 2 legs go through the
    adjoint harmonic transform, matches finite differences."""
    from polybin3d_b200.autograd import bk_numerator
    g = gold("local_los")
    N, L = int(g["N"]), float(g["L"])
    b = quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=list(g["center"]), sightline="local",
              pixel_window="cic", backend="cuda")
    bs = quiet(pb.BSpec, b, g["bedges"], lmax=2, mask=mask24(N, L))
    d = torch.as_tensor(synthetic.lognormal(N, L, seed=21).astype(np.float64), device=b.device)
    num = quiet(bk_numerator, bs, d).cpu().numpy()
    nb = len(num) // 2
    assert rel(num[:nb], g["bk_num"][:nb]) < 1e-10 and rel(num[nb:], g["bk_num"][nb:]) < 1e-10
    check_fd(lambda x: bk_numerator(bs, x), d, bs.N_bins, cubic=True, seed=6, n_vox=4096)
