"""Generate the golden fixtures under tests/golden/ by running the REFERENCE itself.

Run in a container that holds the reference tree (its Python read in place, its Cython
kernels compiled into oracle/_ref/ by oracle/build_ref.sh):

    PB_REFERENCE_ROOT=<directory holding PolyBin3D/> python tests/golden/make_golden.py [case ...]

Every input is regenerated from a seed by polybin3d_b200.synthetic (numpy), so the
fixtures hold only the case parameters and the reference's outputs.  The Monte Carlo
Fisher cases use the reference's own `generate_data(seed)` (legacy MT19937 noise); the
reference's Q-maps are captured by wrapping its integrator object and recording the
map arguments of `cross_integrate` (pspec.py:386) and `integrate_row` (bspec.py:597).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from polybin3d_b200 import synthetic  # noqa: E402
from reference_harness import load_reference  # noqa: E402

CASES = {}


def case(fn):
    CASES[fn.__name__] = fn
    return fn


class _Capture:
    """Proxy around the reference's IntegrationUtils recording Q-map arguments."""

    def __init__(self, inner):
        self._inner = inner
        self.q_rows = []
        self.q_array = None

    def cross_integrate(self, s1, s2, k_edges, l):
        if l == 0:
            self.q_rows.append(np.array(s2))
        return self._inner.cross_integrate(s1, s2, k_edges, l)

    def integrate_row(self, input_map, input_array, kmin, kmax):
        if self.q_array is None:
            self.q_array = np.array(input_array)
        return self._inner.integrate_row(input_map, input_array, kmin, kmax)

    def __getattr__(self, name):
        return getattr(self._inner, name)


def _quiet(fn, *a, **k):
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):
        return fn(*a, **k)


@case
def cfg1(pb):
    """64^3, L=1000, 10 linear bins of width 2kF from kF, no window, FP64 GRF seed 0."""
    N, L = 64, 1000.0
    kF = 2 * np.pi / L
    edges = kF + 2 * kF * np.arange(11)
    data = synthetic.grf(N, L, seed=0)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="none", backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=2)
    pk = _quiet(ps.Pk_ideal, data)
    bs = _quiet(pb.BSpec, base, edges, lmax=0)
    bk = _quiet(bs.Bk_ideal, data)
    out = dict(N=N, L=L, edges=edges, data_seed=0, data_kind="grf", pw="none", pk_lmax=2, bk_lmax=0,
               pk_num=_quiet(ps.Pk_numerator_ideal, data), pk_fish=ps.fish_ideal,
               bk_bins=bs.all_bins, bk_sym=bs.sym_factor, bk_num=_quiet(bs.Bk_numerator_ideal, data),
               bk_fish=bs.fish_ideal)
    for k, v in pk.items():
        out["Pk_" + k] = v
    for k, v in bk.items():
        out["Bk_" + k] = v
    return out


@case
def bk_l2_tsc(pb):
    """32^3, L=500, TSC window, lmax=2, 6 bins to 0.15; float32 lognormal seed 3."""
    N, L = 32, 500.0
    edges = np.linspace(2 * np.pi / L, 0.15, 7)
    data = synthetic.lognormal(N, L, seed=3)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="mkl")
    bs = _quiet(pb.BSpec, base, edges, lmax=2)
    bk = _quiet(bs.Bk_ideal, data)
    out = dict(N=N, L=L, edges=edges, data_seed=3, data_kind="lognormal", pw="tsc", bk_lmax=2,
               bk_bins=bs.all_bins, bk_sym=bs.sym_factor, bk_num=_quiet(bs.Bk_numerator_ideal, data),
               bk_fish=bs.fish_ideal)
    for k, v in bk.items():
        out["Bk_" + k] = v
    bs2 = _quiet(pb.BSpec, base, edges, lmax=2)
    out["bk_fish_nodisc"] = _quiet(bs2.compute_fisher_ideal, discreteness_correction=False)
    return out


@case
def bk_squeeze_partial(pb):
    """24^3, squeezed bins + partial triangles, lmax=0, CIC window, GRF seed 4."""
    N, L = 24, 400.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.12, 4)
    sq = np.concatenate([edges, [0.15, 0.18]])
    data = synthetic.grf(N, L, seed=4)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="mkl")
    bs = _quiet(pb.BSpec, base, edges, lmax=0, k_bins_squeeze=sq, include_partial_triangles=True)
    bk = _quiet(bs.Bk_ideal, data)
    out = dict(N=N, L=L, edges=edges, edges_sq=sq, data_seed=4, data_kind="grf", pw="cic", bk_lmax=0,
               bk_bins=bs.all_bins, bk_sym=bs.sym_factor, bk_num=_quiet(bs.Bk_numerator_ideal, data),
               bk_fish=bs.fish_ideal)
    for k, v in bk.items():
        out["Bk_" + k] = v
    return out


@case
def pk_windows(pb):
    """32^3, L=400, lmax=4, tabulated fiducial P(k), CIC and interlaced-TSC windows."""
    N, L = 32, 400.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.22, 6)
    data = synthetic.lognormal(N, L, seed=7)
    out = dict(N=N, L=L, edges=edges, data_seed=7, data_kind="lognormal", pk_lmax=4)
    for pw in ["cic", "interlaced-tsc"]:
        base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=synthetic.pk_table(1.0), pixel_window=pw, backend="mkl")
        ps = _quiet(pb.PSpec, base, edges, lmax=4)
        pk = _quiet(ps.Pk_ideal, data)
        tag = pw.replace("-", "_")
        out[tag + "_num"] = _quiet(ps.Pk_numerator_ideal, data)
        out[tag + "_fish"] = ps.fish_ideal
        for k, v in pk.items():
            out[tag + "_Pk_" + k] = v
        out[tag + "_fish_nodisc"] = _quiet(ps.compute_fisher_ideal, discreteness_correction=False)
    return out


@case
def grf_noise(pb):
    """generate_data(seed=5, fourier) at 16^3 with a tabulated P(k) and CIC window."""
    N, L = 16, 300.0
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=synthetic.pk_table(1.0), pixel_window="cic", backend="mkl")
    a = base.generate_data(seed=5, output_type="fourier")
    return dict(N=N, L=L, seed=5, pw="cic", a=a)


def _mask24(N, L):
    return synthetic.shell_mask(N, L, r_in=L / 6, r_out=0.4667 * L, n_holes=10, hole_r=(10.0, 30.0),
                                hole_box=0.4667 * L, seed=0)


@case
def pk_fisher_mask(pb):
    """24^3, L=600, lmax=4, 4 bins, shell-sector mask; seeds 0,1; Q-maps of seed 0."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="none", backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=4, mask=mask)
    cap = _Capture(base.integrator)
    base.integrator = cap
    f0 = ps.compute_fisher_contribution(0)
    q0 = np.asarray(cap.q_rows)
    base.integrator = cap._inner
    f1 = ps.compute_fisher_contribution(1)
    fish = 0.5 * (f0 + f1)
    data = (synthetic.lognormal(N, L, seed=11).astype(np.float64) * mask)
    pk = _quiet(ps.Pk_unwindowed, data, fish=fish)
    out = dict(N=N, L=L, edges=edges, pk_lmax=4, f0=f0, f1=f1, q0=q0, data_seed=11,
               num=ps.Pk_numerator(data))
    for k, v in pk.items():
        out["Pk_" + k] = v
    return out


@case
def pk_fisher_nomask(pb):
    """24^3, L=600, lmax=2, 4 bins, no mask, TSC window; seed 2."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=2)
    return dict(N=N, L=L, edges=edges, pk_lmax=2, pw="tsc", f2=ps.compute_fisher_contribution(2))


@case
def bk_fisher_mask(pb):
    """24^3, L=600, lmax=0 and lmax=2, 4 bins, shell-sector mask; seed 0; Q_Ainv of lmax=0."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="none", backend="mkl")
    bs = _quiet(pb.BSpec, base, edges, lmax=0, mask=mask)
    cap = _Capture(base.integrator)
    base.integrator = cap
    f0 = _quiet(bs.compute_fisher_contribution, 0)
    q0 = cap.q_array
    base.integrator = cap._inner
    data = (synthetic.lognormal(N, L, seed=12).astype(np.float64) * mask)
    bk = _quiet(bs.Bk_unwindowed, data, fish=f0 + np.eye(len(f0)) * 0.0, include_linear_term=False)
    bs2 = _quiet(pb.BSpec, base, edges, lmax=2, mask=mask)
    f2 = _quiet(bs2.compute_fisher_contribution, 0)
    out = dict(N=N, L=L, edges=edges, bins0=bs.all_bins, sym0=bs.sym_factor, f0=f0, q0=q0,
               bins2=bs2.all_bins, sym2=bs2.sym_factor, f2_l2=f2, data_seed=12,
               num0=_quiet(bs.Bk_numerator, data, include_linear_term=False))
    for k, v in bk.items():
        out["Bk_" + k] = v
    return out


@case
def bk_fisher_nomask(pb):
    """24^3, L=600, lmax=2, 4 bins, no mask, CIC window; seed 3."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="mkl")
    bs = _quiet(pb.BSpec, base, edges, lmax=2)
    f3 = _quiet(bs.compute_fisher_contribution, 3)
    return dict(N=N, L=L, edges=edges, bk_lmax=2, pw="cic", bins=bs.all_bins, sym=bs.sym_factor, f3=f3)


@case
def bk_linear(pb):
    """24^3, L=600, 4 bins, TSC: Bk_numerator with the linear term.
    (a) lmax=2, shell-sector mask, generate_sims(3), lognormal data seed 13;
    (b) lmax=0, constant mask 0.5, generate_sims(2) with a tabulated P(k), data seed 14;
    (c) lmax=2, shell-sector mask, load_sims of two real-space GRFs (seeds 60, 61) times the mask."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="mkl")
    data = synthetic.lognormal(N, L, seed=13).astype(np.float64) * mask
    bs = _quiet(pb.BSpec, base, edges, lmax=2, mask=mask)
    _quiet(bs.generate_sims, 3)
    num_a = _quiet(bs.Bk_numerator, data)
    out = dict(N=N, L=L, edges=edges, bins=bs.all_bins, sym=bs.sym_factor, num_a=num_a,
               cub_a=_quiet(bs.Bk_numerator, data, include_linear_term=False))
    kt = np.linspace(0.0, 1.0, 400)
    pt = 2e3 * np.exp(-(kt / 0.2) ** 2) + 50.0
    cmask = 0.5 * np.ones((N, N, N))
    data_b = synthetic.lognormal(N, L, seed=14).astype(np.float64) * 0.5
    bs2 = _quiet(pb.BSpec, base, edges, lmax=0, mask=cmask)
    _quiet(bs2.generate_sims, 2, Pk_input=[kt, pt])
    out.update(pk_k=kt, pk_p=pt, bins_b=bs2.all_bins, num_b=_quiet(bs2.Bk_numerator, data_b))
    bs3 = _quiet(pb.BSpec, base, edges, lmax=2, mask=mask)
    _quiet(bs3.load_sims, lambda ii: synthetic.grf(N, L, seed=60 + ii) * mask, 2)
    out.update(num_c=_quiet(bs3.Bk_numerator, data))
    return out


@case
def shot(pb):
    """24^3, L=600, 4 bins, TSC, tabulated positive fiducial P(k): shot-noise contributions.
    PSpec lmax=2 with the shell-sector mask and mask_shot = 0.8 mask (seed 1), PSpec with
    no mask (seed 2); BSpec lmax=2 with the mask and mask_shot = 0.6 mask (seed 1, data =
    lognormal seed 16 times the mask, data2 = 0.7 data; and the cubic-only term)."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    kt = np.linspace(0.0, 1.0, 2000)
    pt = 2e3 * np.exp(-(kt / 0.3) ** 2) + 100.0
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=[kt, pt], pixel_window="tsc", backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=2, mask=mask, mask_shot=0.8 * mask)
    ps2 = _quiet(pb.PSpec, base, edges, lmax=2)
    data = synthetic.lognormal(N, L, seed=16).astype(np.float64) * mask
    bs = _quiet(pb.BSpec, base, edges, lmax=2, mask=mask, mask_shot=0.6 * mask)
    b_full = _quiet(bs.compute_shot_contribution, 1, data=data, data2=0.7 * data)
    b_cub = _quiet(bs.compute_shot_contribution, 1, cubic_only=True)
    return dict(N=N, L=L, edges=edges, pk_k=kt, pk_p=pt, p_mask=_quiet(ps.compute_shot_contribution, 1),
                p_nomask=_quiet(ps2.compute_shot_contribution, 2), bins=bs.all_bins, sym=bs.sym_factor,
                b_full=b_full, b_cubic=b_cub)


@case
def local_los(pb):
    """Local (Yamamoto) line of sight: 32^3, L=500, box centred at (600, 300, 900) Mpc/h, CIC
    window, lognormal data seed 21 times the shell-sector mask.  PSpec lmax=4 (ideal
    numerator and Pk_ideal, S^-1 numerator), BSpec lmax=2 (ideal numerator and Bk_ideal, S^-1
    numerator without the linear term) with 4 bins to 0.15."""
    N, L = 32, 500.0
    center = [600.0, 300.0, 900.0]
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.2, 6)
    bedges = np.linspace(kF, 0.15, 5)
    mask = _mask24(N, L)
    data = synthetic.lognormal(N, L, seed=21).astype(np.float64) * mask
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=center, sightline="local", pixel_window="cic",
                  backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=4, mask=mask)
    pk = _quiet(ps.Pk_ideal, data)
    bs = _quiet(pb.BSpec, base, bedges, lmax=2, mask=mask)
    bk = _quiet(bs.Bk_ideal, data)
    out = dict(N=N, L=L, center=np.asarray(center), edges=edges, bedges=bedges,
               pk_num_ideal=_quiet(ps.Pk_numerator_ideal, data), pk_num=_quiet(ps.Pk_numerator, data),
               pk_fish_ideal=ps.fish_ideal, bk_num_ideal=_quiet(bs.Bk_numerator_ideal, data),
               bk_num=_quiet(bs.Bk_numerator, data, include_linear_term=False), bk_bins=bs.all_bins,
               bk_sym=bs.sym_factor, bk_fish_ideal=bs.fish_ideal)
    for k, v in pk.items():
        out["Pk_" + k] = v
    for k, v in bk.items():
        out["Bk_" + k] = v
    return out


@case
def local_fisher(pb):
    """Local line of sight, Monte Carlo Fisher contributions: 24^3, L=600, box centred at
    (700, 400, 900) Mpc/h, TSC window, 4 bins; Pk lmax=4 and Bk lmax=2, each with the
    shell-sector mask (seed 0) and a constant mask 0.7 (seed 1)."""
    N, L = 24, 600.0
    center = [700.0, 400.0, 900.0]
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=center, sightline="local", pixel_window="tsc",
                  backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=4, mask=mask)
    f0 = _quiet(ps.compute_fisher_contribution, 0)
    ps2 = _quiet(pb.PSpec, base, edges, lmax=4, mask=0.7 * np.ones((N, N, N)))
    f1 = _quiet(ps2.compute_fisher_contribution, 1)
    bs = _quiet(pb.BSpec, base, edges, lmax=2, mask=mask)
    bf0 = _quiet(bs.compute_fisher_contribution, 0)
    bs2 = _quiet(pb.BSpec, base, edges, lmax=2, mask=0.7 * np.ones((N, N, N)))
    bf1 = _quiet(bs2.compute_fisher_contribution, 1)
    return dict(N=N, L=L, center=np.asarray(center), edges=edges, f0=f0, f1=f1, bk_bins=bs.all_bins,
                bk_sym=bs.sym_factor, bf0=bf0, bf1=bf1)


@case
def local_shot(pb):
    """Local line of sight, shot-noise contributions: 24^3, L=600, box centred at
    (700, 400, 900) Mpc/h, TSC window, tabulated positive P(k), 4 bins; PSpec lmax=4 with the
    shell-sector mask and mask_shot = 0.8 mask (seed 1); BSpec lmax=2 with mask_shot =
    0.6 mask (seed 1, data = lognormal seed 16 times the mask, data2 = 0.7 data)."""
    N, L = 24, 600.0
    center = [700.0, 400.0, 900.0]
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    kt = np.linspace(0.0, 1.0, 2000)
    pt = 2e3 * np.exp(-(kt / 0.3) ** 2) + 100.0
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=[kt, pt], boxcenter=center, sightline="local",
                  pixel_window="tsc", backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=4, mask=mask, mask_shot=0.8 * mask)
    data = synthetic.lognormal(N, L, seed=16).astype(np.float64) * mask
    bs = _quiet(pb.BSpec, base, edges, lmax=2, mask=mask, mask_shot=0.6 * mask)
    b_full = _quiet(bs.compute_shot_contribution, 1, data=data, data2=0.7 * data)
    return dict(N=N, L=L, center=np.asarray(center), edges=edges, pk_k=kt, pk_p=pt,
                p_mask=_quiet(ps.compute_shot_contribution, 1), bins=bs.all_bins, sym=bs.sym_factor, b_full=b_full)


@case
def pk_cov_theory(pb):
    """PSpec (global sightline) covariance and theory-matrix contributions: 24^3, L=600, CIC
    window, lmax=4, 4 bins.  Covariance with Pk_cov = [k, P0, P2] (shell-sector mask,
    mask_shot = 0.5 mask, seed 2; constant mask 0.7, seed 3); theory matrix with 6 theory
    bins to 0.12 and lmax_theory = 4 (mask, seed 4).  Local sightline (box centred at
    (700, 400, 900) Mpc/h, TSC window, lmax=2): covariance with [k, P0, P2] (mask, mask_shot =
    0.5 mask, seed 5), theory matrix with lmax_theory = 4 (seed 6), covariance with [k, P0]
    and the constant mask 0.7 (seed 7)."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    kt = np.linspace(0.0, 1.0, 2000)
    p0 = 3e3 * np.exp(-(kt / 0.25) ** 2) + 200.0
    p2 = 800.0 * np.exp(-(kt / 0.2) ** 2)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=4, mask=mask, mask_shot=0.5 * mask)
    c2 = _quiet(ps.compute_covariance_contribution, 2, [kt, p0, p2])
    ps2 = _quiet(pb.PSpec, base, edges, lmax=4, mask=0.7 * np.ones((N, N, N)))
    c3 = _quiet(ps2.compute_covariance_contribution, 3, [kt, p0, p2])
    kth = np.linspace(kF, 0.12, 7)
    f4, t4 = _quiet(ps.compute_theory_contribution, 4, kth, lmax_theory=4)
    center = [700.0, 400.0, 900.0]
    lbase = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=center, sightline="local", pixel_window="tsc",
                   backend="mkl")
    lps = _quiet(pb.PSpec, lbase, edges, lmax=2, mask=mask, mask_shot=0.5 * mask)
    lc5 = _quiet(lps.compute_covariance_contribution, 5, [kt, p0, p2])
    lf6, lt6 = _quiet(lps.compute_theory_contribution, 6, kth, lmax_theory=4)
    lps2 = _quiet(pb.PSpec, lbase, edges, lmax=2, mask=0.7 * np.ones((N, N, N)))
    lc7 = _quiet(lps2.compute_covariance_contribution, 7, [kt, p0])
    return dict(N=N, L=L, edges=edges, pk_k=kt, p0=p0, p2=p2, c2=c2, c3=c3, kth=kth, f4=f4, t4=t4,
                center=np.asarray(center), lc5=lc5, lf6=lf6, lt6=lt6, lc7=lc7)


@case
def bk_cov(pb):
    """BSpec covariance contributions: 24^3, L=600, 4 bins, lmax=2, Pk_cov = [k, P0, P2].
    Global sightline, CIC window: shell-sector mask with mask_shot = 0.5 mask (seed 2; the
    caution printed for the shared shot mask), the same mask with mask_shot_2pt = 0.8 mask
    (seed 3), constant mask 0.7 with [k, P0] (seed 4; mask_shot_2pt given, as the
    reference needs one there).  Local sightline (box centred at (700, 400, 900) Mpc/h,
    TSC window): shell-sector mask, mask_shot = 0.5 mask (seed 5)."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    kt = np.linspace(0.0, 1.0, 2000)
    p0 = 3e3 * np.exp(-(kt / 0.25) ** 2) + 200.0
    p2 = 800.0 * np.exp(-(kt / 0.2) ** 2)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="mkl")
    bs = _quiet(pb.BSpec, base, edges, lmax=2, mask=mask, mask_shot=0.5 * mask)
    c2 = _quiet(bs.compute_covariance_contribution, 2, [kt, p0, p2])
    c3 = _quiet(bs.compute_covariance_contribution, 3, [kt, p0, p2], mask_shot_2pt=0.8 * mask)
    bs2 = _quiet(pb.BSpec, base, edges, lmax=2, mask=0.7 * np.ones((N, N, N)))
    c4 = _quiet(bs2.compute_covariance_contribution, 4, [kt, p0], mask_shot_2pt=np.ones((N, N, N)))
    center = [700.0, 400.0, 900.0]
    lbase = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=center, sightline="local", pixel_window="tsc",
                   backend="mkl")
    lbs = _quiet(pb.BSpec, lbase, edges, lmax=2, mask=mask, mask_shot=0.5 * mask)
    lc5 = _quiet(lbs.compute_covariance_contribution, 5, [kt, p0, p2])
    return dict(N=N, L=L, edges=edges, pk_k=kt, p0=p0, p2=p2, bins=bs.all_bins, sym=bs.sym_factor, c2=c2, c3=c3,
                c4=c4, center=np.asarray(center), lsym=lbs.sym_factor, lc5=lc5)


@case
def integral_constraints(pb):
    """Integral constraints in the Monte Carlo matrices: 24^3, L=600, 4 bins, CIC window,
    shell-sector mask, mask_IC = (mask > 0).  Global sightline with the global constraint:
    PSpec lmax=2 Fisher (seed 0), covariance with [k, P0, P2] and mask_shot = 0.5 mask
    (seed 1), theory matrix lmax_theory = 4 (seed 2); BSpec lmax=2 Fisher (seed 0),
    covariance (seed 1), Bk_numerator with the linear term from generate_sims(2) (lognormal
    data seed 13).  Local sightline (box centred at (700, 400, 900) Mpc/h) with the radial
    constraint in |r| shells [1300, 1360, 1410, 1450, 1700) Mpc/h (mask voxels below 1300
    give 0): PSpec lmax=2 Fisher (seed 3), BSpec lmax=2 Fisher (seed 2)."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    mask_ic = (mask > 0).astype(np.float64)
    kt = np.linspace(0.0, 1.0, 2000)
    p0 = 3e3 * np.exp(-(kt / 0.25) ** 2) + 200.0
    p2 = 800.0 * np.exp(-(kt / 0.2) ** 2)
    kth = np.linspace(kF, 0.12, 7)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=2, mask=mask, mask_shot=0.5 * mask, add_GIC=True, mask_IC=mask_ic)
    out = dict(N=N, L=L, edges=edges, pk_k=kt, p0=p0, p2=p2, kth=kth)
    out["pf0"] = _quiet(ps.compute_fisher_contribution, 0)
    out["pc1"] = _quiet(ps.compute_covariance_contribution, 1, [kt, p0, p2])
    out["pf2"], out["pt2"] = _quiet(ps.compute_theory_contribution, 2, kth, lmax_theory=4)
    bs = _quiet(pb.BSpec, base, edges, lmax=2, mask=mask, mask_shot=0.5 * mask, add_GIC=True, mask_IC=mask_ic)
    out["bf0"] = _quiet(bs.compute_fisher_contribution, 0)
    out["bc1"] = _quiet(bs.compute_covariance_contribution, 1, [kt, p0, p2])
    out["bins"], out["sym"] = bs.all_bins, bs.sym_factor
    data = synthetic.lognormal(N, L, seed=13).astype(np.float64) * mask
    _quiet(bs.generate_sims, 2)
    out["bnum"] = _quiet(bs.Bk_numerator, data)
    out["bcub"] = _quiet(bs.Bk_numerator, data, include_linear_term=False)
    center = [700.0, 400.0, 900.0]
    redges = np.array([1300.0, 1360.0, 1410.0, 1450.0, 1700.0])
    lbase = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=center, sightline="local", pixel_window="cic",
                   backend="mkl")
    lps = _quiet(pb.PSpec, lbase, edges, lmax=2, mask=mask, add_RIC=True, mask_IC=mask_ic, radial_bins_RIC=redges)
    out["lpf3"] = _quiet(lps.compute_fisher_contribution, 3)
    lbs = _quiet(pb.BSpec, lbase, edges, lmax=2, mask=mask, add_RIC=True, mask_IC=mask_ic, radial_bins_RIC=redges)
    out["lbf2"] = _quiet(lbs.compute_fisher_contribution, 2)
    out.update(center=np.asarray(center), redges=redges, lsym=lbs.sym_factor)
    return out


@case
def local_odd(pb):
    """Local line of sight with odd multipoles (odd_l=True, lmax=3): 24^3, L=600, box centred
    at (700, 400, 900) Mpc/h, TSC window, tabulated positive P(k), 4 bins, shell-sector mask
    with mask_shot = 0.8 mask.  Pk_numerator and Pk_numerator_ideal of lognormal data
    (seed 21) times the mask, the Fisher contribution (seed 0), the shot-noise contribution
    (seed 1), the theory matrix with odd_l (lmax_theory = 4, seed 2); and with lmax=2 (even)
    the theory matrix with the wide-angle terms (lmax_theory = 4, seed 3)."""
    N, L = 24, 600.0
    center = [700.0, 400.0, 900.0]
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    kth = np.linspace(kF, 0.12, 7)
    mask = _mask24(N, L)
    kt = np.linspace(0.0, 1.0, 2000)
    pt = 3e3 * np.exp(-(kt / 0.25) ** 2) + 200.0
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, Pk=[kt, pt], boxcenter=center, sightline="local",
                  pixel_window="tsc", backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=3, mask=mask, mask_shot=0.8 * mask, odd_l=True)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * mask
    out = dict(N=N, L=L, center=np.asarray(center), edges=edges, kth=kth, pk_k=kt, pk_p=pt)
    out["num"] = _quiet(ps.Pk_numerator, d)
    out["num_ideal"] = _quiet(ps.Pk_numerator_ideal, d)
    out["f0"] = _quiet(ps.compute_fisher_contribution, 0)
    out["shot1"] = _quiet(ps.compute_shot_contribution, 1)
    out["tf2"], out["tt2"] = _quiet(ps.compute_theory_contribution, 2, kth, lmax_theory=4)
    ps2 = _quiet(pb.PSpec, base, edges, lmax=2, mask=mask)
    out["wf3"], out["wt3"] = _quiet(ps2.compute_theory_contribution, 3, kth, lmax_theory=4, include_wideangle=True)
    return out


def sinv_pair(base, N):
    """A non-trivial, non-symmetric S^-1 for the custom-weighting fixture: S^-1 x =
    IFT[w(k) FT[u x]] with w(k) = 1/(1 + (|k|/0.05)^2) and u = 1 + 0.5 sin(2 pi i0/N) along
    the first grid axis; its transpose is u IFT[w(k) FT[x]].  Both take and return real maps
    or half spectra as the reference's applySinv does."""
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


@case
def custom_sinv(pb):
    """PSpec with a user S^-1 (sinv_pair): 24^3, L=600, 4 bins, shell-sector mask with
    mask_shot = 0.5 mask, lognormal data (seed 21) times the mask.  (a) global, CIC window,
    lmax=2: numerator, Fisher (seed 0), shot noise (seed 1), covariance with [k, P0, P2]
    (seed 2), theory matrix lmax_theory = 4 (seed 3); (b) constant mask 0.7: numerator,
    Fisher (seed 4), covariance with [k, P0] (seed 5); (c) local sightline (box centred at
    (700, 400, 900) Mpc/h), no window, lmax=2: numerator, Fisher (seed 6), shot noise (seed
    7); (d) applySinv alone (taken as its own transpose), global, Fisher (seed 8)."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    kth = np.linspace(kF, 0.12, 7)
    mask = _mask24(N, L)
    kt = np.linspace(0.0, 1.0, 2000)
    p0 = 3e3 * np.exp(-(kt / 0.25) ** 2) + 200.0
    p2 = 800.0 * np.exp(-(kt / 0.2) ** 2)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * mask
    out = dict(N=N, L=L, edges=edges, kth=kth, pk_k=kt, p0=p0, p2=p2)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="mkl")
    si, st = sinv_pair(base, N)
    ps = _quiet(pb.PSpec, base, edges, lmax=2, mask=mask, mask_shot=0.5 * mask, applySinv=si, applySinv_transpose=st)
    out["a_num"] = _quiet(ps.Pk_numerator, d)
    out["a_f0"] = _quiet(ps.compute_fisher_contribution, 0)
    out["a_s1"] = _quiet(ps.compute_shot_contribution, 1)
    out["a_c2"] = _quiet(ps.compute_covariance_contribution, 2, [kt, p0, p2])
    out["a_f3"], out["a_t3"] = _quiet(ps.compute_theory_contribution, 3, kth, lmax_theory=4)
    cm = 0.7 * np.ones((N, N, N))
    ps2 = _quiet(pb.PSpec, base, edges, lmax=2, mask=cm, applySinv=si, applySinv_transpose=st)
    out["b_num"] = _quiet(ps2.Pk_numerator, synthetic.lognormal(N, L, seed=21).astype(np.float64) * 0.7)
    out["b_f4"] = _quiet(ps2.compute_fisher_contribution, 4)
    out["b_c5"] = _quiet(ps2.compute_covariance_contribution, 5, [kt, p0])
    center = [700.0, 400.0, 900.0]
    lbase = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, boxcenter=center, sightline="local", backend="mkl")
    lsi, lst = sinv_pair(lbase, N)
    lps = _quiet(pb.PSpec, lbase, edges, lmax=2, mask=mask, mask_shot=0.5 * mask, applySinv=lsi,
                 applySinv_transpose=lst)
    out["c_num"] = _quiet(lps.Pk_numerator, d)
    out["c_f6"] = _quiet(lps.compute_fisher_contribution, 6)
    out["c_s7"] = _quiet(lps.compute_shot_contribution, 7)
    ps4 = _quiet(pb.PSpec, base, edges, lmax=2, mask=mask, applySinv=si)
    out["d_f8"] = _quiet(ps4.compute_fisher_contribution, 8)
    out["center"] = np.asarray(center)
    return out


@case
def bk_custom_sinv(pb):
    """BSpec with a user S^-1 (sinv_pair): 24^3, L=600, 4 bins, lmax=2, CIC window,
    shell-sector mask with mask_shot = 0.5 mask, lognormal data (seed 21) times the mask:
    numerator without and with the linear term (generate_sims(2)), Fisher (seed 0),
    shot noise with data2 = 0.7 data (seed 1), covariance with [k, P0, P2] (seed 2); and the
    constant mask 0.7: numerator, Fisher (seed 3)."""
    N, L = 24, 600.0
    kF = 2 * np.pi / L
    edges = np.linspace(kF, 0.11, 5)
    mask = _mask24(N, L)
    kt = np.linspace(0.0, 1.0, 2000)
    p0 = 3e3 * np.exp(-(kt / 0.25) ** 2) + 200.0
    p2 = 800.0 * np.exp(-(kt / 0.2) ** 2)
    d = synthetic.lognormal(N, L, seed=21).astype(np.float64) * mask
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="cic", backend="mkl")
    si, st = sinv_pair(base, N)
    bs = _quiet(pb.BSpec, base, edges, lmax=2, mask=mask, mask_shot=0.5 * mask, applySinv=si, applySinv_transpose=st)
    out = dict(N=N, L=L, edges=edges, pk_k=kt, p0=p0, p2=p2, bins=bs.all_bins)
    out["cub"] = _quiet(bs.Bk_numerator, d, include_linear_term=False)
    out["sym"] = bs.sym_factor
    _quiet(bs.generate_sims, 2)
    out["num"] = _quiet(bs.Bk_numerator, d)
    out["f0"] = _quiet(bs.compute_fisher_contribution, 0)
    out["s1"] = _quiet(bs.compute_shot_contribution, 1, data=d, data2=0.7 * d)
    out["c2"] = _quiet(bs.compute_covariance_contribution, 2, [kt, p0, p2])
    bs2 = _quiet(pb.BSpec, base, edges, lmax=2, mask=0.7 * np.ones((N, N, N)), applySinv=si, applySinv_transpose=st)
    out["b_cub"] = _quiet(bs2.Bk_numerator, synthetic.lognormal(N, L, seed=21).astype(np.float64) * 0.7,
                          include_linear_term=False)
    out["b_f3"] = _quiet(bs2.compute_fisher_contribution, 3)
    return out


def _sparse(m):
    """Nonzero entries of a matrix as (rows, cols, values) (the ideal Fisher matrices couple
    only the multipoles of one triangle bin, so they are block-sparse)."""
    r, c = np.nonzero(m)
    return r.astype(np.int32), c.astype(np.int32), m[r, c]


def _survey_mask(N, L):
    """The shell-sector mask of the 128^3 Monte Carlo Fisher workloads: 250 < r < 700 Mpc/h,
    octant x,y,z > 0, 200 holes of radius 5-20 Mpc/h (seed 0)."""
    return synthetic.shell_mask(N, L, r_in=250.0, r_out=700.0, n_holes=200, hole_r=(5.0, 20.0), hole_box=700.0,
                                seed=0)


@case
def cfg2_bk256(pb):
    """The headline: Bk_ideal at 256^3, L=2000, TSC, lmax=2, 16 linear bins 2pi/2000..0.2,
    float32 lognormal seed 0.  Numerator, symmetry factors, ideal Fisher (sparse) and b0/b2."""
    N, L = 256, 2000.0
    edges = np.linspace(2 * np.pi / L, 0.2, 17)
    data = synthetic.lognormal(N, L, seed=0)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="tsc", backend="mkl")
    bs = _quiet(pb.BSpec, base, edges, lmax=2)
    t = time.time()
    num = _quiet(bs.Bk_numerator_ideal, data)
    t_num = time.time() - t
    t = time.time()
    bk = _quiet(bs.Bk_ideal, data)
    fr, fc, fv = _sparse(bs.fish_ideal)
    out = dict(N=N, L=L, edges=edges, data_seed=0, data_kind="lognormal", pw="tsc", bk_lmax=2,
               bk_bins=bs.all_bins, bk_sym=bs.sym_factor, bk_num=num, fish_rows=fr, fish_cols=fc, fish_vals=fv,
               fish_n=bs.fish_ideal.shape[0], t_num=t_num, t_fisher=time.time() - t)
    for k, v in bk.items():
        out["Bk_" + k] = v
    return out


@case
def cfg3_pk128(pb):
    """Monte Carlo Pk Fisher at 128^3, L=1500, lmax=4, 20 linear bins 2pi/1500..0.25, the
    survey mask: compute_fisher_contribution(0) (60 x 60) and the numerator of the masked
    lognormal field (seed 31)."""
    N, L = 128, 1500.0
    edges = np.linspace(2 * np.pi / L, 0.25, 21)
    mask = _survey_mask(N, L)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="none", backend="mkl")
    ps = _quiet(pb.PSpec, base, edges, lmax=4, mask=mask)
    t = time.time()
    f0 = _quiet(ps.compute_fisher_contribution, 0)
    t_f = time.time() - t
    data = synthetic.lognormal(N, L, seed=31).astype(np.float64) * mask
    return dict(N=N, L=L, edges=edges, pk_lmax=4, f0=f0, t_fisher=t_f, data_seed=31,
                num=_quiet(ps.Pk_numerator, data))


@case
def cfg4_bk128(pb):
    """Monte Carlo Bk Fisher at 128^3, L=1500, lmax=0, 12 linear bins 2pi/1500..0.2, the
    survey mask: compute_fisher_contribution(0) (203 x 203), the symmetry factors and the
    cubic numerator of the masked lognormal field (seed 41)."""
    N, L = 128, 1500.0
    edges = np.linspace(2 * np.pi / L, 0.2, 13)
    mask = _survey_mask(N, L)
    base = _quiet(pb.PolyBin3D, [L] * 3, [N] * 3, pixel_window="none", backend="mkl")
    bs = _quiet(pb.BSpec, base, edges, lmax=0, mask=mask)
    t = time.time()
    f0 = _quiet(bs.compute_fisher_contribution, 0)
    t_f = time.time() - t
    data = synthetic.lognormal(N, L, seed=41).astype(np.float64) * mask
    return dict(N=N, L=L, edges=edges, bk_lmax=0, bins=bs.all_bins, sym=bs.sym_factor, f0=f0, t_fisher=t_f,
                data_seed=41, num=_quiet(bs.Bk_numerator, data, include_linear_term=False))


def main(names=None):
    pb = load_reference()
    for name, fn in CASES.items():
        if names and name not in names:
            continue
        t = time.time()
        out = fn(pb)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **{k: np.asarray(v) for k, v in out.items()})
        print("%-22s %6.1fs  %8.1f KB" % (name, time.time() - t, os.path.getsize(path) / 1024))


if __name__ == "__main__":
    main(sys.argv[1:])
