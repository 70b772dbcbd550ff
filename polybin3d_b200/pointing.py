"""Pointing matrix of a spatially varying mask, with optional integral constraints.

The Monte Carlo matrices apply the survey window P to simulated fields (PolyBin3D/pspec.py:
199-213, bspec.py:412-427).  Without constraints P is the mask.  The global integral
constraint (pointing_GIC, cython/utils.pyx:405-424) removes from each map its mean over the
unweighted mask mask_IC before the mask multiplies it; the radial one (pointing_RIC,
utils.pyx:448-481) removes the mean over each shell of |r| instead, and sets voxels in no
shell to 0.  The transposes (utils.pyx:426-446, 483-516) multiply by the mask and subtract
mask_IC times the (shell) mean of mask x map, normalised by the same mask_IC sums.

Maps come in batches (R, n0, n1, n2) on the device: the plain mask is one elementwise
launch; the constraints add one weighted reduction per map (a matrix-vector product for
the global mean, an index-add over shell indices for the radial means) and one fused
broadcast.
"""
import numpy as np
import torch

from . import _native as nat


class Pointing:
    """P and P^dag of one estimator's mask: kind 'mask', 'GIC' or 'RIC'."""

    def __init__(self, base, mask, mask_IC=None, kind='mask', radial_edges=None):
        self.base = base
        self.kind = kind
        self.mask = mask
        self._typed = {}
        if kind == 'mask':
            return
        dev = base.device
        mic = np.asarray(mask_IC, dtype=np.float64)
        self.mask_ic = torch.as_tensor(np.ascontiguousarray(mic), device=dev)
        if kind == 'GIC':
            self.norm = float(mic.sum())
            return
        r = base.r_grids
        modr = np.sqrt(r[0] ** 2. + r[1] ** 2. + r[2] ** 2.)
        edges = np.asarray(radial_edges, dtype=np.float64)
        zidx = np.full(modr.shape, -1, dtype=np.int64)
        for iz in range(len(edges) - 1):
            zidx[(modr >= edges[iz]) & (modr < edges[iz + 1])] = iz
        self.nz = len(edges) - 1
        # shell index + 1 per voxel (0: outside every shell), and the mask_IC sum of each shell
        self.zidx1 = torch.as_tensor((zidx + 1).reshape(-1), device=dev)
        self.inside = torch.as_tensor((zidx >= 0), device=dev)
        den = np.bincount(zidx[zidx >= 0], weights=mic[zidx >= 0], minlength=self.nz)
        self.den = torch.as_tensor(den, device=dev)

    def _as(self, t, dtype):
        if t.dtype == dtype:
            return t
        key = (id(t), dtype)
        if key not in self._typed:
            self._typed[key] = t.to(dtype)
        return self._typed[key]

    def __call__(self, x, transpose=False, out=None):
        """P x (or P^dag x) for real maps x (..., n0, n1, n2); `out` may alias x."""
        b = self.base
        m = self._as(self.mask, x.dtype)
        if self.kind == 'mask':
            return nat.elementwise(nat.PB_EW_MUL, x, m, out=out, y_period=b.nreal)
        mic = self._as(self.mask_ic, x.dtype)
        shape = x.shape
        xf = x.reshape(-1, b.nreal)
        w = (m if transpose else mic).reshape(-1)
        if self.kind == 'GIC':
            av = (xf @ w) / self.norm
            res = m.reshape(1, -1) * xf - mic.reshape(1, -1) * av[:, None] if transpose \
                else m.reshape(1, -1) * (xf - av[:, None])
        else:
            num = torch.zeros((xf.shape[0], self.nz + 1), dtype=x.dtype, device=x.device)
            num.index_add_(1, self.zidx1, xf * w.reshape(1, -1))
            av = torch.cat([torch.zeros_like(num[:, :1]), num[:, 1:] / self._as(self.den, x.dtype)], 1)
            avv = av[:, self.zidx1]
            res = m.reshape(1, -1) * xf - mic.reshape(1, -1) * avv if transpose \
                else m.reshape(1, -1) * (xf - avv)
            res = torch.where(self.inside.reshape(1, -1), res, torch.zeros_like(res))
        res = res.reshape(shape)
        if out is None:
            return res
        out.copy_(res)
        return out
