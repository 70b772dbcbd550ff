"""Real spherical harmonics for the local (Yamamoto) line of sight.

Multipoles about a line of sight that changes from voxel to voxel use the addition theorem
sum_m Y_lm(k^) Y_lm(r^) = L_l(k^ . r^): the Fourier transform of Y_lm(r^) a(r), weighted by
Y_lm(k^) and summed over m, gives the l-th multipole of a about the line of sight to each
voxel (PolyBin3D/base.py:402-411, apply_fourier_harmonics).  The harmonic grids of the
positions (full grid) and of the wavevectors (half grid) are made once on the host and kept
on the device.
"""
import numpy as np
import torch

from . import _native as nat


def real_harmonics(k_grids, l):
    """Real spherical harmonics of the unit vector for l = 1..4 (odd l: the odd_l set); the
    same functions and normalisation as compute_real_harmonics
    (PolyBin3D/cython/utils.pyx:518-609), so that sum_m Y_lm(k) Y_lm(k') = L_l(k.k')."""
    kx, ky, kz = k_grids
    norm = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    safe = np.where(norm == 0, 1.0, norm)
    xh, yh, zh = [np.where(norm == 0, 0.0, c / safe) for c in (kx, ky, kz)]
    if l == 1:
        return [yh, zh, xh]
    if l == 3:
        return [(45. * xh ** 2 * yh - 15. * yh ** 3) * np.sqrt(1. / 360.),
                (30. * xh * yh * zh) * np.sqrt(1. / 60.),
                (-1.5 * xh ** 2 * yh - 1.5 * yh ** 3 + 6. * yh * zh ** 2) * np.sqrt(1. / 6.),
                (-1.5 * xh ** 2 * zh - 1.5 * yh ** 2 * zh + zh ** 3),
                (-1.5 * xh ** 3 - 1.5 * xh * yh ** 2 + 6. * xh * zh ** 2) * np.sqrt(1. / 6.),
                (15. * xh ** 2 * zh - 15. * yh ** 2 * zh) * np.sqrt(1. / 60.),
                (15. * xh ** 3 - 45. * xh * yh ** 2) * np.sqrt(1. / 360.)]
    if l == 2:
        return [6.0 * xh * yh * np.sqrt(1.0 / 12.0),
                3.0 * yh * zh * np.sqrt(1.0 / 3.0),
                zh ** 2 - xh ** 2 / 2.0 - yh ** 2 / 2.0,
                3.0 * xh * zh * np.sqrt(1.0 / 3.0),
                (3 * xh ** 2 - 3 * yh ** 2) * np.sqrt(1.0 / 12.0)]
    if l == 4:
        x2, y2, z2 = xh * xh, yh * yh, zh * zh
        return [(420.0 * x2 * xh * yh - 420.0 * xh * y2 * yh) * np.sqrt(1.0 / 20160.0),
                (315.0 * x2 * yh * zh - 105.0 * y2 * yh * zh) * np.sqrt(1.0 / 2520.0),
                (-15.0 * x2 * xh * yh - 15.0 * xh * y2 * yh + 90.0 * xh * yh * z2) * np.sqrt(1.0 / 180.0),
                (-7.5 * x2 * yh * zh - 7.5 * y2 * yh * zh + 10.0 * yh * z2 * zh) * np.sqrt(1.0 / 10.0),
                35.0 / 8.0 * z2 * z2 - 15.0 / 4.0 * z2 + 3.0 / 8.0,
                (-7.5 * x2 * xh * zh - 7.5 * xh * y2 * zh + 10.0 * xh * z2 * zh) * np.sqrt(1.0 / 10.0),
                (-7.5 * x2 * x2 + 45.0 * x2 * z2 + 7.5 * y2 * y2 - 45.0 * y2 * z2) * np.sqrt(1.0 / 180.0),
                (105.0 * x2 * xh * zh - 315.0 * xh * y2 * zh) * np.sqrt(1.0 / 2520.0),
                (105.0 * x2 * x2 - 630.0 * x2 * y2 + 105.0 * y2 * y2) * np.sqrt(1.0 / 20160.0)]
    raise ValueError("l must be 1, 2, 3 or 4")


class Harmonics:
    """Device harmonic grids of one box for the multipoles 1..4, and their use."""

    def __init__(self, base):
        self.base = base
        self._grids = {}

    def _grid(self, kind, l, dtype):
        key = (kind, l, dtype)
        g = self._grids.get(key)
        if g is None:
            b = self.base
            coords = b.r_grids if kind == 'r' else b.k_grids
            g = torch.as_tensor(np.ascontiguousarray(np.asarray(real_harmonics(coords, l))), dtype=dtype,
                                device=b.device)
            self._grids[key] = g
        return g

    def apply_fourier(self, a_real, l):
        """sum_m Y_lm(k) rfftn(Y_lm(r) a(r)) as a half spectrum of a_real's precision: the
        2l+1 products in one elementwise launch, one batched r2c, the m-sum on the device."""
        b = self.base
        yr = self._grid('r', l, a_real.dtype)
        yk = self._grid('k', l, a_real.dtype)
        prod = nat.elementwise(nat.PB_EW_MUL, yr, a_real.contiguous(), y_period=b.nreal)
        b.n_FFTs_forward += yr.shape[0]
        F = b.fft_r2c(prod)
        return (F * yk).sum(0)
