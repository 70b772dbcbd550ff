"""Gaussian-covariance filter shared by the PSpec and BSpec covariance contributions.

The Monte Carlo covariance of the unwindowed estimators (PolyBin3D/pspec.py:149-162,
PolyBin3D/bspec.py:447-471) reruns the Fisher computation with every S^-1 P replaced by
S^-1 [P xi P^dag + N] S^-dag: xi is the correlation function of a model power spectrum
Pk_cov applied as a Fourier-space weight (plus, for the local line of sight, the
harmonic transforms of its l > 0 multipoles; base.py:413-437), P the mask and N the shot
mask.  With the trivial S^-1 this is, on a block of maps held as half spectra:

* constant mask m: the diagonal weight m^2 xi(k) + m;
* varying mask: P IFT[xi FT[P^dag x]] + mask_shot x, x the real-space map and P the mask
  (with an integral constraint, its pointing matrix).

Every step is a batched spectral filter, cuFFT transform or elementwise product on the
device; the maps of a block go through each step together.
"""
import numpy as np
import torch

from . import _native as nat


def xi_grids(base, Pk_cov):
    """Device grids of Pk_cov = [k, P0(, P2(, P4))] keyed by multipole (pspec.py:241-252,
    bspec.py:481-496): global sightline, one grid P0 + L2(mu) P2 + L4(mu) P4; local, one
    grid per multipole.  Linear interpolation in |k|, zero outside the table."""
    from scipy.interpolate import interp1d
    from scipy.special import legendre
    Pk_cov = np.asarray(Pk_cov, dtype=np.float64)
    terms = [interp1d(Pk_cov[0], Pk_cov[i], bounds_error=False, fill_value=0.)(base.modk_grid)
             for i in range(1, len(Pk_cov))]
    if base.sightline == 'global':
        g = terms[0]
        for i, t in enumerate(terms[1:]):
            g = g + legendre(2 * (i + 1))(base.muk_grid) * t
        grids = {0: g}
    else:
        grids = {2 * i: t for i, t in enumerate(terms)}
    return {l: torch.as_tensor(np.ascontiguousarray(v, dtype=np.float64), device=base.device)
            for l, v in grids.items()}


def xi_real(base, X, x_real, xi):
    """apply_xi with real output (base.py:413-437) for a block of maps: X (R, half) half
    spectra, x_real (R, n0, n1, n2) the same maps in real space.  P0 X, plus for each local
    multipole l > 0 one half of P_l sum_m Y_lm(k) FT[Y_lm(r) x] and one half of
    sum_m Y_lm(r) IFT[Y_lm(k) P_l X]."""
    grid, F64, nh = base.grid, nat.PB_F64, base.nhalf
    invN = 1.0 / base.nreal
    nrow = X.shape[0]
    P = torch.empty_like(X)
    nat.spectral_filter(grid, F64, X, P, [(i, -1.0, np.inf, 0, 0, invN, 1) for i in range(nrow)], w=xi[0],
                        src_stride=nh)
    ells = sorted(xi)[1:]
    harm = base.harmonics if ells else None
    for l in ells:
        for i in range(nrow):
            H = harm.apply_fourier(x_real[i], l)
            nat.spectral_filter(grid, F64, H[None], P, [(0, -1.0, np.inf, 0, 0, 0.5 * invN, 1)], w=xi[l],
                                accumulate=True, dst=[i])
    base.n_FFTs_reverse += nrow
    out = base.fft_c2r(P)
    for l in ells:
        yr = harm._grid('r', l, torch.float64)
        yk = harm._grid('k', l, torch.float64)
        for mi in range(yr.shape[0]):
            nat.spectral_filter(grid, F64, X, P, [(i, -1.0, np.inf, 0, 0, 0.5 * invN, 1) for i in range(nrow)],
                                w=(yk[mi] * xi[l]).contiguous(), src_stride=nh)
            base.n_FFTs_reverse += nrow
            out.addcmul_(base.fft_c2r(P), yr[mi])
    return out


def cov_rows(base, R, xi, const_mask, mask_mean, point, mask_shot, real=None):
    """R <- S^-1 [P xi P^dag + N] S^-dag of a block of maps, trivial S^-1 (pspec.py:277-290,
    307-323; bspec.py:499-519).  R (R, half) holds the half spectra, multiplied by 1/N^3
    beforehand for a varying mask; `real` optional real-space maps added to them.  point:
    the pointing matrix (`pointing.Pointing`: P, and P^dag with transpose=True), mask_shot
    the device shot mask (varying mask only).  Returns R."""
    nrow = R.shape[0]
    if const_mask:
        if len(xi) > 1:
            raise ValueError("local multipoles of Pk_cov need a varying mask (the reference applies xi "
                             "without a real-space map for a constant mask)")
        if real is not None:
            base.n_FFTs_forward += nrow
            R.add_(base.fft_r2c(real))
        mm = float(mask_mean)
        w = (xi[0] * (mm * mm) + mm).contiguous()
        nat.spectral_filter(base.grid, nat.PB_F64, R, R, [(i, -1.0, np.inf, 0, 0, 1.0, 1) for i in range(nrow)],
                            w=w, src_stride=base.nhalf)
        return R
    base.n_FFTs_reverse += nrow
    sid = base.fft_c2r(R)
    if real is not None:
        sid.add_(real)
    t = point(sid, True)
    base.n_FFTs_forward += nrow
    u = xi_real(base, base.fft_r2c(t, out=R), t, xi)
    point(u, False, out=u)
    u.add_(nat.elementwise(nat.PB_EW_MUL, sid, mask_shot, out=t, y_period=base.nreal))
    base.n_FFTs_forward += nrow
    return base.fft_r2c(u, out=R)


def cov_custom(base, x, real, xi, const_mask, mask_mean, point, mask_shot, sinv, sinv_t):
    """S^-1 [P xi P^dag + N] S^-dag of one map with a caller's S^-1 (pspec.py:277-290,
    307-323; bspec.py:507-518): sinv / sinv_t(x, input_type, output_type) apply S^-1 and
    S^-dag; x a real map if `real`, else a half spectrum; returns a half spectrum."""
    it = 'real' if real else 'fourier'
    if const_mask:
        if len(xi) > 1:
            raise ValueError("local multipoles of Pk_cov need a varying mask (the reference applies xi "
                             "without a real-space map for a constant mask)")
        sid = sinv_t(x, it, 'fourier')
        mm = float(mask_mean)
        return sinv(sid * (xi[0] * (mm * mm) + mm), 'fourier', 'fourier')
    sid = sinv_t(x, it, 'real')
    t = point(sid, True)
    base.n_FFTs_forward += 1
    u = xi_real(base, base.fft_r2c(t)[None], t[None], xi)[0]
    return sinv(point(u, False) + sid * mask_shot, 'real', 'fourier')
