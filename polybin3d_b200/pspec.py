"""Power-spectrum estimators, backend='cuda' (mirrors PolyBin3D/pspec.py, global sightline).

Numerators: one r2c, an optional weighting pass, and one k-bin x Legendre reduction
for all multipoles at once (pb_bin_reduce).  Monte Carlo Fisher: GRF from the reference's
own noise draw, the N_bins Q-maps batched through one filter launch and batched FFTs,
and every Fisher row from one CROSS reduction (FP64 throughout).
"""
import numpy as np
import torch

from . import _native as nat
from . import covariance
from . import pointing
from . import autotune
from . import realisations


class PSpec:
    """Power spectrum estimators (pspec.py:10-26 for the inputs)."""

    def __init__(self, base, k_bins, lmax=2, mask=None, applySinv=None, odd_l=False, add_GIC=False, mask_IC=None,
                 add_RIC=False, radial_bins_RIC=[], mask_shot=None, applySinv_transpose=None, *, verb=True):
        self.base = base
        self.applySinv = applySinv
        self.k_bins = np.asarray(k_bins)
        self.lmax = lmax
        self.Nk = len(k_bins) - 1
        self.odd_l = odd_l
        self.Nl = self.lmax + 1 if self.odd_l else self.lmax // 2 + 1
        self.Nl_even = self.lmax // 2 + 1
        self.N_bins = self.Nk * self.Nl
        self.add_GIC = add_GIC
        self.add_RIC = add_RIC
        self.applySinv_transpose = applySinv_transpose

        if verb:
            print("")
        # range checks (pspec.py:46-59)
        assert np.max(self.k_bins) < np.min(base.kNy), "k_max must be less than k_Nyquist!"
        assert np.min(self.k_bins) >= np.max(base.kF), "k_min must be at least the k_fundamental!"
        assert np.max(self.k_bins) <= base.Pfid[0][-1], "Fiducial power spectrum should extend up to k_max!"
        assert np.min(self.k_bins) >= base.Pfid[0][0], "Fiducial power spectrum should extend down to k_min!"
        if verb:
            print("Binning: %d bins in [%.3f, %.3f] h/Mpc" % (self.Nk, np.min(self.k_bins), np.max(self.k_bins)))
            print("l-max: %d" % (self.lmax))
        if self.odd_l:
            assert self.lmax > 0, "lmax must be greater than 0 to use odd harmonics!"
            assert self.base.sightline == 'local', "Odd spherical harmonics should only be used for local line-of-sight!"
        assert type(self.lmax) == int, "l-max must be an integer!"
        assert self.lmax <= 4, "Only l-max<=4 is currently supported!"
        if not np.all(np.diff(self.k_bins) > 0):
            raise ValueError("k_bins must be strictly increasing")

        # mask (pspec.py:62-85)
        if type(mask) == type(None):
            self.const_mask = True
            self.mask_mean = 1.
            self.sq_mask_mean = 1.
            assert not self.add_GIC, "Global integral constraint cannot be used without a mask!"
            assert not self.add_RIC, "Radial integral constraint cannot be used without a mask!"
        else:
            if type(mask) != np.ndarray:
                mask = np.array(mask.cpu() if isinstance(mask, torch.Tensor) else mask)
            self.mask = mask.astype(np.float64)
            if type(mask_IC) != type(None):
                self.mask_IC = mask_IC.astype(np.float64)
            if np.std(self.mask) < 1e-12:
                self.const_mask = True
                self.mask_mean = np.mean(self.mask)
            else:
                self.const_mask = False
            self.sq_mask_mean = np.mean(self.mask ** 2)
        if verb:
            print("Mask: constant" if self.const_mask else "Mask: spatially varying")
        if type(mask_shot) != type(None):
            self.mask_shot = mask_shot.astype(np.float64)

        # S^-1 (pspec.py:92-99): the trivial filter, or the caller's, applied to device maps
        # (a real map or a half spectrum in, either out); its transpose defaults to itself
        self._custom_sinv = self.applySinv is not None
        if self._custom_sinv and type(self.applySinv_transpose) != type(lambda x: x):
            self.applySinv_transpose = self.applySinv
            if verb:
                print("## Caution: assuming S^-1 is Hermitian!")
        # integral constraints (pspec.py:101-111)
        if self.add_GIC:
            if verb:
                print("Accounting for global integral constraint")
            assert hasattr(self, 'mask_IC'), "Need to supply mask_IC!"
        if self.add_RIC:
            assert not self.add_GIC, "Radial integral constraint imposes global integral constraint automatically!"
            assert hasattr(self, 'mask_IC'), "Need to supply mask_IC!"
            assert len(radial_bins_RIC) > 0, "Radial bins need to be supplied for radial integral constraint!"
            if verb:
                print("Accounting for radial integral constraint across %d bins" % (len(radial_bins_RIC) - 1))
            self.radial_bins_RIC = np.asarray(radial_bins_RIC, dtype=np.float64)
        self._pt = None
        if not self._custom_sinv:
            self.applySinv = self.base.applySinv_trivial
            self.applySinv_transpose = self.base.applySinv_trivial
        self._captured = {}

    def _ylm(self, kind):
        """Real harmonics of positions ('r') or wavevectors ('k') by l, as the reference's
        Ylm_real / Ylm_fourier (pspec.py:86-91): FP64 device grids, made on first use and
        shared with the ones the local-sightline multipoles use; None unless the sightline
        is local and lmax > 0."""
        if self.base.sightline != 'local' or self.lmax == 0:
            return None
        ls = range(1, self.lmax + 1) if self.odd_l else range(2, self.lmax + 1, 2)
        return {l: self.base.harmonics._grid(kind, l, torch.float64) for l in ls}

    @property
    def Ylm_real(self):
        return self._ylm('r')

    @property
    def Ylm_fourier(self):
        return self._ylm('k')

    def get_ks(self):
        """Central k of each bin (pspec.py:122-128)."""
        return np.asarray([0.5 * (self.k_bins[b] + self.k_bins[b + 1]) for b in range(self.Nk)])

    # ------------------------------------------------------------------------------
    # helpers
    # ------------------------------------------------------------------------------
    def _ells(self, Nl):
        return [(2 * li, 0) for li in range(Nl)]

    def _data_device(self, data, dtype=None):
        if not isinstance(data, torch.Tensor):
            assert type(data[0, 0, 0]) in [np.float32, np.float64], "Data must be of type float32 or float64!"
        else:
            assert data.dtype in (torch.float32, torch.float64), "Data must be of type float32 or float64!"
        return self.base.as_device(data, dtype)

    def _weighted_spectrum(self, data, filtering, dtype=None):
        """x(k) = rfftn(d) / W [* invP / sqrt(<m^2>)] on the device (pspec.py:617-640)."""
        b = self.base
        x = self._data_device(data, dtype)
        xk = b.to_fourier(x)
        prec = nat.precision_of(xk.dtype)
        rd = torch.float64 if prec == nat.PB_F64 else torch.float32
        if filtering == 'ideal':
            unit = b._unit_pk and b.pixel_window == 'none'
            if not unit:
                w = b.to_device_grid('pk_ideal_w', lambda: self._ideal_weight(), rd)
                nat.spectral_filter(b.grid, prec, xk, xk, [(0, -1.0, np.inf, 0, 0, 1.0, 1)], w=w)
            scale = 1.0 / self.sq_mask_mean
        else:
            if b.pixel_window != 'none':
                w = b.to_device_grid('window', lambda: b.pixel_window_grid, rd)
                nat.spectral_filter(b.grid, prec, xk, xk, [(0, -1.0, np.inf, 0, 0, 1.0, -1)], w=w)
            if self._custom_sinv:                                        # pspec.py:629-640
                y = self._sinv(xk, 'fourier', 'fourier') if b.pixel_window != 'none' else \
                    self._sinv(x, 'real', 'fourier')
                xk = y.to(xk.dtype)
            scale = 1.0
        return xk, scale

    def _sinv(self, x, input_type, output_type, transpose=False):
        """The caller's S^-1 (or S^-dag) on one device map (pspec.py:92-99); the result as
        a contiguous FP64 device tensor (half spectrum or real map)."""
        f = self.applySinv_transpose if transpose else self.applySinv
        y = f(x, input_type=input_type, output_type=output_type)
        if not isinstance(y, torch.Tensor):
            y = torch.as_tensor(np.ascontiguousarray(y))
        dt = torch.complex128 if output_type == 'fourier' else torch.float64
        return y.to(device=self.base.device, dtype=dt).contiguous()

    def _dagger_custom(self, x, real, xi=None):
        """(S^-1 P)^dag x with the caller's S^-dag (pspec.py:291-305), or its covariance form
        S^-1 [P xi P^dag + N] S^-dag (307-323), for one map: x a real map if `real`, else a
        half spectrum; returns a half spectrum."""
        b = self.base
        it = 'real' if real else 'fourier'
        if xi is None:
            if self.const_mask:
                return self._sinv(x, it, 'fourier', transpose=True) * float(self.mask_mean)
            r = self._sinv(x, it, 'real', transpose=True)
            b.n_FFTs_forward += 1
            return b.fft_r2c(self._pointing()(r, True))
        if self.const_mask:
            sid = self._sinv(x, it, 'fourier', transpose=True)
            if len(xi) > 1:
                raise ValueError("local multipoles of Pk_cov need a varying mask (the reference applies xi "
                                 "without a real-space map for a constant mask)")
            mm = float(self.mask_mean)
            return self._sinv(sid * (xi[0] * (mm * mm) + mm), 'fourier', 'fourier')
        sid = self._sinv(x, it, 'real', transpose=True)
        t = self._pointing()(sid, True)
        b.n_FFTs_forward += 1
        u = covariance.xi_real(b, b.fft_r2c(t)[None], t[None], xi)[0]
        ms = b.to_device_grid(('pk_mask_shot', id(self)), lambda: self.mask_shot, torch.float64)
        u = self._pointing()(u, False) + sid * ms
        return self._sinv(u, 'real', 'fourier')

    def _ideal_weight(self):
        b = self.base
        w = b.invPk0_grid.copy()
        if b.pixel_window != 'none':
            W = b.pixel_window_grid
            nz = W != 0
            w[nz] = w[nz] / W[nz]
            w[~nz] = 0.
        return w

    def _compute_pk_numerator(self, data, filtering='ideal'):
        """Numerator (pspec.py:613-686): the ideal one has the even multipoles only."""
        assert filtering in ['ideal', 'Sinv'], "Unknown filtering option supplied!"
        b = self.base
        xk, s2 = self._weighted_spectrum(data, filtering)
        Nl = self.Nl if filtering == 'Sinv' else self.Nl_even
        out = torch.empty(Nl * self.Nk, dtype=torch.float64, device=b.device)
        scale = 0.5 * s2 * b.volume / float(b.gridsize.prod()) ** 2
        prec = nat.precision_of(xk.dtype)
        if b.sightline == 'global' or Nl == 1:
            nat.bin_reduce(b.grid, prec, nat.PB_RED_ABS2, xk, None, 1, self.k_bins, self._ells(Nl), scale, out, b.ws)
            return out.cpu().numpy()
        # local sightline (pspec.py:643-680): the monopole as above; multipole l is the
        # binned cross spectrum of x with sum_m Y_lm(k) FT[Y_lm(r) x(r)], times -i for odd l
        # (odd_l, S^-1 numerator only) so that it is real
        odd = self.odd_l and filtering == 'Sinv'
        Nk = self.Nk
        nat.bin_reduce(b.grid, prec, nat.PB_RED_ABS2, xk, None, 1, self.k_bins, [(0, 0)], scale, out[:Nk], b.ws)
        x_real = b.to_real(xk)
        for li in range(1, Nl):
            l = li * (2 - odd)
            lm = b.harmonics.apply_fourier(x_real, l)
            if l % 2:
                lm = lm * (-1j)
            nat.bin_reduce(b.grid, prec, nat.PB_RED_CROSS, xk, lm, 1, self.k_bins, [(0, 0)], scale,
                           out[li * Nk:(li + 1) * Nk], b.ws)
        return out.cpu().numpy()

    # ------------------------------------------------------------------------------
    # unwindowed estimator
    # ------------------------------------------------------------------------------
    def Pk_numerator(self, data):
        """Numerator of the unwindowed estimator, trivial S^-1 (pspec.py:131-139)."""
        if not self.const_mask:
            assert data.shape == self.mask.shape, "Data must have same shape as the mask!"
        return self._compute_pk_numerator(data, filtering='Sinv')

    def _mask_device(self):
        return self.base.to_device_grid(('pk_mask', id(self)), lambda: self.mask, torch.float64)

    def _pointing(self):
        """The pointing matrix of the varying mask, with the integral constraint asked for."""
        if self._pt is None:
            kind = 'RIC' if self.add_RIC else ('GIC' if self.add_GIC else 'mask')
            self._pt = pointing.Pointing(self.base, self._mask_device(), getattr(self, 'mask_IC', None), kind,
                                         getattr(self, 'radial_bins_RIC', None))
        return self._pt

    def _fisher_from_fields(self, a, xi=None, theory=None):
        """Fisher contributions of a batch of GRFs a (B, half) complex128 (pspec.py:215-493).
        xi: device grids of the covariance spectrum (covariance contributions: every S^-1 P
        becomes S^-1 [P xi P^dag + N] S^-dag); theory: (k_bins_theory, Nl_theory), which adds
        the binning matrix of each realisation, (B, N_bins, Nl_theory * Nk_theory)."""
        b = self.base
        B = a.shape[0]
        nh = b.nhalf
        grid = b.grid
        F64 = nat.PB_F64
        invN = 1.0 / b.nreal
        ainv_w = b.to_device_grid('ainv', b._ainv_weight, torch.float64)
        Ainv = torch.empty_like(a)
        nat.spectral_filter(grid, F64, a, Ainv, [(i, -1.0, np.inf, 0, 0, 1.0, 1) for i in range(B)], w=ainv_w,
                            src_stride=nh)
        bm = None
        if theory is not None:
            k_th, nl_th = theory[:2]
            bm = torch.zeros((B, self.N_bins, nl_th * (len(k_th) - 1)), dtype=torch.float64, device=b.device)
        if self._custom_sinv:
            # the caller's S^-1, one map at a time as the reference applies it (pspec.py:270-290)
            SinvP = torch.empty_like(a)
            for i in range(B):
                if xi is not None:
                    SinvP[i] = self._dagger_custom(a[i] if self.const_mask else b.to_real(a[i]), not self.const_mask,
                                                   xi)
                elif self.const_mask:
                    SinvP[i] = self._sinv(a[i], 'fourier', 'fourier') * float(self.mask_mean)
                else:
                    SinvP[i] = self._sinv(self._pointing()(b.to_real(a[i]), False), 'real', 'fourier')
            qscale = 1.0
        elif xi is not None:
            # S^-1 P a -> S^-1 [P xi P^dag + N] S^-dag a (pspec.py:270-290, 330-332)
            SinvP = a.clone()
            if not self.const_mask:
                nat.spectral_filter(grid, F64, SinvP, SinvP, [(i, -1.0, np.inf, 0, 0, invN, 0) for i in range(B)],
                                    src_stride=nh)
            SinvP = self._cov_rows(SinvP, xi)
            qscale = 1.0
        elif self.const_mask:
            SinvP = a
            qscale = self.mask_mean * self.mask_mean
        else:
            ar = a.clone()
            nat.spectral_filter(grid, F64, ar, ar, [(i, -1.0, np.inf, 0, 0, invN, 0) for i in range(B)],
                                src_stride=nh)
            ar = b.fft_c2r(ar)
            b.n_FFTs_reverse += B
            self._pointing()(ar, False, out=ar)
            SinvP = b.fft_r2c(ar)
            b.n_FFTs_forward += B
            qscale = 1.0
        fish = torch.empty((B, self.N_bins, self.N_bins), dtype=torch.float64, device=b.device)
        scaling = 0.5 * b.volume / float(b.gridsize.prod()) ** 2
        if b.sightline == 'local' and (self.Nl > 1 or theory is not None):
            for i in range(B):
                S = SinvP[i] * self.mask_mean if (self.const_mask and xi is None and not self._custom_sinv) \
                    else SinvP[i]
                self._fisher_local(Ainv[i], S, scaling, fish[i], xi=xi, theory=theory,
                                   bm=None if bm is None else bm[i])
            return fish if theory is None else (fish, bm)
        rows = [(li, ki) for li in range(self.Nl) for ki in range(self.Nk)]
        for i in range(B):
            Q = torch.empty((self.N_bins,) + b.nhalf_shape, dtype=torch.complex128, device=b.device)
            qs = 1.0 if self._custom_sinv else (qscale if self.const_mask else invN)
            maps = [(i, self.k_bins[ki], self.k_bins[ki + 1], 2 * li, 0, qs, 0) for (li, ki) in rows]
            nat.spectral_filter(grid, F64, SinvP, Q, maps, src_stride=nh)
            if self._custom_sinv:
                for r in range(self.N_bins):
                    Q[r] = self._dagger_custom(Q[r], False, xi)
            elif xi is not None:
                Q = self._cov_rows(Q, xi)
            elif not self.const_mask:
                qr = b.fft_c2r(Q)
                b.n_FFTs_reverse += self.N_bins
                self._pointing()(qr, True, out=qr)
                Q = b.fft_r2c(qr, out=Q)
                b.n_FFTs_forward += self.N_bins
            autotune.bin_reduce(grid, F64, nat.PB_RED_CROSS, Ainv[i], Q, self.N_bins, self.k_bins,
                                self._ells(self.Nl), scaling, fish[i], b.ws)
            if theory is not None:                                       # pspec.py:395-402
                autotune.bin_reduce(grid, F64, nat.PB_RED_CROSS, Ainv[i], Q, self.N_bins, theory[0],
                                    self._ells(theory[1]), scaling, bm[i], b.ws)
        return fish if theory is None else (fish, bm)

    def _xi_grids(self, Pk_cov):
        return covariance.xi_grids(self.base, Pk_cov)

    def _cov_rows(self, R, xi, real=None):
        ms = None if self.const_mask else self.base.to_device_grid(('pk_mask_shot', id(self)),
                                                                   lambda: self.mask_shot, torch.float64)
        return covariance.cov_rows(self.base, R, xi, self.const_mask, getattr(self, 'mask_mean', None),
                                   None if self.const_mask else self._pointing(), ms, real)

    def _fisher_local(self, Ainv, S, scaling, fish, xi=None, theory=None, bm=None):
        """One realisation's Fisher rows for the local sightline (pspec.py:334-366, 380-438,
        440-486).  With H_l[x] = sum_m Y_lm(k) FT[Y_lm(r) IFT x] and D = (S^-1 P)^dag:
        monopole rows Q = D Theta_b S; multipole rows
        Q = 1/2 D Theta_b H_l[S] + 1/2 D sum_m Y_lm(r) IFT[Theta_b Y_lm(k) S], both parts
        times -i for odd l (odd_l); column block 0 is the binned cross spectrum of Q with
        A^-1 a, block l the one of i Q (odd l) or Q with H_l[A^-1 a].  All rows of a
        multipole go through each step as one batch.  With xi, D is the covariance form
        S^-1 [P xi P^dag + N] S^-dag.  theory = (k_bins_theory, Nl_theory, lmax_theory,
        wide-angle, odd multipoles): the binning matrix bm gets the same cross spectra in the
        theory bins; with the wide-angle terms the odd-l maps H_l[A^-1 a / |r|] add to the
        l = 2, 4 blocks with the per-bin coefficients of pspec.py:424-438."""
        b = self.base
        grid, F64, Nk = b.grid, nat.PB_F64, self.Nk
        invN = 1.0 / b.nreal
        harm = b.harmonics
        Q = torch.empty((self.N_bins,) + b.nhalf_shape, dtype=torch.complex128, device=b.device)
        mm = float(self.mask_mean) if self.const_mask else 1.0

        def dagger_rows(R, real=None):
            """R <- D R for a block of rows whose Fourier part R (already scaled by 1/N^3 for
            a varying mask, by the mask mean for a constant one) may come with a real-space
            part `real` (unnormalised, added before the mask)."""
            if self._custom_sinv:
                # the caller's S^-dag: each part of each row on its own (pspec.py:466-483)
                for r in range(R.shape[0]):
                    q = self._dagger_custom(R[r], False, xi)
                    if real is not None:
                        q = q + self._dagger_custom(real[r], True, xi)
                    R[r] = q
                return R
            if xi is not None:
                return self._cov_rows(R, xi, real)
            if self.const_mask:
                if real is not None:
                    R.add_(b.fft_r2c(real), alpha=mm)
                    b.n_FFTs_forward += R.shape[0]
                return R
            rr = b.fft_c2r(R)
            b.n_FFTs_reverse += R.shape[0]
            if real is not None:
                rr.add_(real)
            self._pointing()(rr, True, out=rr)
            b.n_FFTs_forward += R.shape[0]
            return b.fft_r2c(rr, out=R)

        qs = 1.0 if self._custom_sinv else (invN if not self.const_mask else (1.0 if xi is not None else mm))
        bands = [(0, self.k_bins[ki], self.k_bins[ki + 1], 0, 0, qs, 0) for ki in range(Nk)]
        nat.spectral_filter(grid, F64, S, Q[:Nk], bands)
        dagger_rows(Q[:Nk])
        S_real = b.to_real(S)
        for li in range(1, self.Nl):
            l = li * (2 - self.odd_l)
            R = Q[li * Nk:(li + 1) * Nk]
            nat.spectral_filter(grid, F64, harm.apply_fourier(S_real, l), R,
                                [(0, lo, hi, 0, 0, 0.5 * sc, 0) for (_, lo, hi, _, _, sc, _) in bands])
            if l % 2:
                R.mul_(-1j)
            yr = harm._grid('r', l, torch.float64)
            yk = harm._grid('k', l, torch.float64)
            real_map = torch.zeros((Nk,) + tuple(int(n) for n in b.gridsize), dtype=torch.float64, device=b.device)
            T = torch.empty((Nk,) + b.nhalf_shape, dtype=torch.complex128, device=b.device)
            for mi in range(yr.shape[0]):
                nat.spectral_filter(grid, F64, S, T, [(0, lo, hi, 0, 0, 0.5 * invN, 1) for (_, lo, hi, _, _, _, _) in bands],
                                    w=yk[mi])
                if l % 2:
                    T.mul_(-1j)
                t = b.fft_c2r(T)
                b.n_FFTs_reverse += Nk
                real_map.addcmul_(t, yr[mi])
            dagger_rows(R, real_map)
        leg_cache = {}
        A_real = b.to_real(Ainv) if (self.Nl > 1 or theory is not None) else None

        def leg(l, over_r=False):
            """H_l[A^-1 a] (or of A^-1 a / |r|), times -i for odd l: its cross spectrum with Q
            is the one of H_l with i Q (pspec.py:409-413, 418-421)."""
            key = (l, over_r)
            if key not in leg_cache:
                x = A_real
                if over_r:                                               # div_real (utils.pyx:265-278)
                    r = b.to_device_grid('modr', lambda: np.sqrt(b.r_grids[0] ** 2. + b.r_grids[1] ** 2.
                                                                 + b.r_grids[2] ** 2.), torch.float64)
                    x = torch.where(r != 0, A_real / torch.where(r != 0, r, torch.ones_like(r)),
                                    torch.zeros_like(r))
                h = harm.apply_fourier(x, l)
                leg_cache[key] = h * (-1j) if l % 2 else h
            return leg_cache[key]

        def cross(a, edges):
            out = torch.empty((self.N_bins, len(edges) - 1), dtype=torch.float64, device=b.device)
            autotune.bin_reduce(grid, F64, nat.PB_RED_CROSS, a, Q, self.N_bins, edges, [(0, 0)], scaling, out,
                                b.ws)
            return out

        fish[:, :Nk] = cross(Ainv, self.k_bins)
        for li in range(1, self.Nl):
            fish[:, li * Nk:(li + 1) * Nk] = cross(leg(li * (2 - self.odd_l)), self.k_bins)
        if theory is None:
            return fish
        k_th, nl_th, lmax_th, wide, odd_t = theory
        nkt = len(k_th) - 1
        bm.zero_()
        bm[:, :nkt] = cross(Ainv, k_th)
        if not wide:
            for li in range(1, nl_th):
                bm[:, li * nkt:(li + 1) * nkt] = cross(leg(li * (2 - odd_t)), k_th)
            return fish
        # wide-angle terms (pspec.py:424-438): even l as usual; odd l from A^-1 a / |r| with
        # coefficient i alpha_b per theory bin, Re(i alpha s1 s2*) = alpha Re((i s1) s2*)
        kfac = torch.as_tensor(self.derivative_coefficient(k_th), device=b.device)
        for l in range(1, lmax_th + 1):
            if l % 2 == 0:
                bm[:, l // 2 * nkt:(l // 2 + 1) * nkt] += cross(leg(l), k_th)
                continue
            terms = []
            if l == 1 and lmax_th >= 2:
                terms.append((1, 3.0 / 5.0 * (3 + kfac)))
            if l == 3 and lmax_th >= 2:
                terms.append((1, 3.0 / 5.0 * (2 - kfac)))
            if l == 3 and lmax_th >= 4:
                terms.append((2, 10.0 / 9.0 * (5 + kfac)))
            if terms:
                c = cross(leg(l, over_r=True) * (-1.0), k_th)    # leg carries -i: (-1)(-i) = i
                for blk, alpha in terms:
                    bm[:, blk * nkt:(blk + 1) * nkt] += c * alpha[None, :]
        return fish

    @staticmethod
    def derivative_coefficient(k):
        """Coefficients of the numerical k dP/dk over the theory bins (pspec.py:368-378)."""
        nk = len(k) - 1
        kfac = np.zeros(nk)
        for ki in range(nk):
            if 0 < ki - 1 < nk - 1:
                kfac[ki] += k[ki - 1] / (k[ki] - k[ki - 2])
            if 0 < ki + 1 < nk - 1:
                kfac[ki] -= k[ki + 1] / (k[ki + 2] - k[ki])
            kfac[ki] += k[0] / (k[1] - k[0]) * ((ki == 1) - (ki == 0))
            kfac[ki] -= k[-1] / (k[-1] - k[-2]) * ((ki == nk - 1) - (ki == nk - 2))
        return kfac

    def compute_fisher_contribution(self, seed, verb=False):
        """Fisher contribution of one GRF with the reference's noise for this seed (pspec.py:141-147)."""
        b = self.base
        re, im = b.reference_noise(seed + int(1e7))
        a = b.grf_from_noise(torch.as_tensor(re, device=b.device)[None], torch.as_tensor(im, device=b.device)[None])
        return self._fisher_from_fields(a)[0].cpu().numpy()

    def compute_fisher(self, N_it, verb=False, *, batch=4, group=None, noise='reference'):
        """Mean Fisher over seeds 0..N_it-1 (pspec.py:553-569); `batch` GRFs per device pass.
        Under an initialised torch.distributed process group (`group`, default the world)
        the seeds are shared round-robin over the ranks; every rank returns the same
        matrix, summed in seed order exactly as the one-process loop sums it.
        noise='reference': the reference's own MT19937 draw per seed (identical inputs);
        noise='philox': white noise drawn on the device (Philox, keyed by seed + 1e7) and
        each batch of realisations replayed from one captured CUDA graph."""
        assert noise in ('reference', 'philox'), "noise must be 'reference' or 'philox'"
        b = self.base
        feed = None
        if noise == 'reference' and realisations.prefetch_pays(N_it, b.gridsize):
            # the reference's draws for this rank's seeds, made ahead on host workers
            rank, size = realisations.world(group)
            feed = realisations.noise_pool(b.gridsize).stream(
                [s + int(1e7) for s in realisations.seeds_of_rank(N_it, rank, size)])

        def contrib(seeds):
            if noise == 'philox' and self._custom_sinv:
                # a caller's S^-1 may synchronise or allocate on the host: no graph capture
                return self._fisher_from_fields(b.grf_philox(np.asarray(seeds, dtype=np.int64) + int(1e7)))
            if noise == 'philox':
                cap = self._captured.get(batch)
                if cap is None:
                    cap = realisations.CapturedBatch(
                        lambda sd: self._fisher_from_fields(b.grf_philox(sd + int(1e7))), batch, b)
                    self._captured[batch] = cap
                return cap.run(seeds)
            if feed is not None:
                nre, nim = feed.take(len(seeds), b.device)
            else:
                noise_ = [b.reference_noise(s + int(1e7)) for s in seeds]
                nre = torch.as_tensor(np.stack([n[0] for n in noise_]), device=b.device)
                nim = torch.as_tensor(np.stack([n[1] for n in noise_]), device=b.device)
            return self._fisher_from_fields(b.grf_from_noise(nre, nim))

        def progress(seeds):
            for s in seeds:
                if s % 5 == 0 or verb:
                    print("Computing Fisher contribution %d of %d" % (s + 1, N_it))

        fish = realisations.mc_mean(contrib, N_it, (self.N_bins, self.N_bins), b.device, batch=batch, group=group,
                                    progress=progress)
        fish = fish.cpu().numpy()
        self.fish = fish
        self.inv_fish = np.linalg.inv(fish)
        return fish

    def Pk_unwindowed(self, data, fish=[], shot_num=[], subtract_shotnoise=False):
        """Unwindowed estimator (pspec.py:571-611)."""
        if len(fish) != 0:
            self.fish = fish
            self.inv_fish = np.linalg.inv(fish)
        if len(shot_num) != 0 or subtract_shotnoise:
            self.shot_num = shot_num
            self.shot = np.matmul(self.inv_fish, self.shot_num)
        if not hasattr(self, 'inv_fish'):
            raise Exception("Need to compute Fisher matrix first!")
        if not hasattr(self, 'shot') and subtract_shotnoise:
            raise Exception("Need to compute shot-noise first!")
        Pk_num = self.Pk_numerator(data)
        Pk_out = np.matmul(self.inv_fish, Pk_num)
        if subtract_shotnoise:
            Pk_out -= self.shot
        Pk_dict = {}
        index = 0
        for l in range(0, self.lmax + 1, 2 - self.odd_l):
            Pk_dict['p%s' % l] = Pk_out[index:index + self.Nk]
            index += self.Nk
        return Pk_dict

    # ------------------------------------------------------------------------------
    # ideal estimator
    # ------------------------------------------------------------------------------
    def Pk_numerator_ideal(self, data):
        """Numerator of the ideal estimator (pspec.py:689-700)."""
        if not self.const_mask:
            assert data.shape == self.mask.shape, "Data must have same shape as the mask!"
        return self._compute_pk_numerator(data, filtering='ideal')

    def compute_fisher_ideal(self, discreteness_correction=True, Pk_fid='default'):
        """Ideal Fisher matrix (pspec.py:702-752), FP64 reductions on the device."""
        b = self.base
        print("Computing ideal Fisher matrix")
        fish = np.zeros((self.Nl_even * self.Nk, self.Nl_even * self.Nk))
        if Pk_fid != 'default':
            if (np.asarray(Pk_fid) == None).all() or (Pk_fid == 'none'):  # noqa: E711
                k_tmp = np.arange(np.min(b.kF) / 10., np.max(b.kNy) * 2, np.min(b.kF) / 10.)
                Pfid = np.asarray([k_tmp, 1. + 0. * k_tmp])
            else:
                assert len(Pk_fid) == 2, "Pk should contain k and P_0(k) columns"
                Pfid = np.asarray(Pk_fid)
            from scipy.interpolate import interp1d
            Pk0 = interp1d(Pfid[0], Pfid[1], bounds_error=False, fill_value=0.)(b.modk_grid)
            inv = np.zeros(b.modk_grid.shape)
            good = (Pk0 != 0) & np.isfinite(Pk0)
            inv[good] = 1. / Pk0[good]
            w = torch.as_tensor(inv, device=b.device)
        else:
            w = None if b._unit_pk else b.to_device_grid('invPk0', lambda: b.invPk0_grid, torch.float64)
        if discreteness_correction:
            pairs = [(2 * la, 2 * lb) for la in range(self.Nl_even) for lb in range(self.Nl_even)]
        else:
            pairs = [(0, 0)]
        out = torch.empty(len(pairs) * self.Nk, dtype=torch.float64, device=b.device)
        nat.bin_reduce(b.grid, nat.PB_F64, nat.PB_RED_REAL2, w, None, 1, self.k_bins, pairs, 0.5, out, b.ws)
        vals = out.cpu().numpy().reshape(len(pairs), self.Nk)
        if discreteness_correction:
            for e, (la2, lb2) in enumerate(pairs):
                la, lb = la2 // 2, lb2 // 2
                fish[la * self.Nk:(la + 1) * self.Nk, lb * self.Nk:(lb + 1) * self.Nk] = np.diag(vals[e])
        else:
            for la in range(self.Nl_even):
                fish[la * self.Nk:(la + 1) * self.Nk, la * self.Nk:(la + 1) * self.Nk] = np.diag(vals[0]) / (4. * la + 1.)
        self.fish_ideal = fish
        self.inv_fish_ideal = np.linalg.inv(self.fish_ideal)
        return fish

    def Pk_ideal(self, data, fish_ideal=[], discreteness_correction=True):
        """Ideal estimator (pspec.py:754-784)."""
        if len(fish_ideal) != 0:
            self.fish_ideal = fish_ideal
            self.inv_fish_ideal = np.linalg.inv(fish_ideal)
        if not hasattr(self, 'inv_fish_ideal'):
            self.compute_fisher_ideal(discreteness_correction=discreteness_correction)
        Pk_num_ideal = self.Pk_numerator_ideal(data)
        Pk_out = np.matmul(self.inv_fish_ideal, Pk_num_ideal)
        Pk_dict = {}
        index = 0
        for l in range(0, self.lmax + 1, 2):
            Pk_dict['p%s' % l] = Pk_out[index:index + self.Nk]
            index += self.Nk
        return Pk_dict

    def compute_shot_contribution(self, seed):
        """Shot-noise contribution of one GRF (pspec.py:495-549): a is drawn
        with spectrum P_A = 1/P_fid (pixel window included), A^-1 = (1/P_A) / W^2, and the
        k-binned cross spectrum of S^-1 a with S^-1 N A^-1 a (N: mask_shot, or the mask mean
        for a constant mask) is halved and normalised by V / N^6."""
        if not self.const_mask:
            assert hasattr(self, 'mask_shot'), "Must supply mask_shot to compute shot-noise contribution"
        b = self.base
        dev = b.device
        F64 = nat.PB_F64
        PkA = [b.Pfid[0], 1. / b.Pfid[1]]
        if getattr(self, '_invPA', None) is None:
            self._invPA = self._shot_inv_pa(PkA)
        invPA = self._invPA
        re, im = b.reference_noise(seed + int(1e7))
        a = b.grf_from_noise(torch.as_tensor(re, device=dev), torch.as_tensor(im, device=dev), Pk_input=PkA)
        sna = b.applyAinv(a, invPk0_grid=invPA, input_type='fourier',
                          output_type='fourier' if self.const_mask else 'real')
        scale = 0.5 * b.volume / float(b.gridsize.prod()) ** 2
        if self._custom_sinv:                                            # pspec.py:514-522
            if self.const_mask:
                sna = self._sinv(sna, 'fourier', 'fourier') * float(self.mask_mean)
            else:
                m = b.to_device_grid(('pk_mask_shot', id(self)), lambda: self.mask_shot, torch.float64)
                sna = self._sinv(sna * m, 'real', 'fourier')
            a = self._sinv(a, 'fourier', 'fourier')
        elif self.const_mask:
            scale *= self.mask_mean
        else:
            m = b.to_device_grid(('pk_mask_shot', id(self)), lambda: self.mask_shot, torch.float64)
            nat.elementwise(nat.PB_EW_MUL, sna, m, out=sna, y_period=b.nreal)
            sna = b.to_fourier(sna)
        out = torch.empty(self.N_bins, dtype=torch.float64, device=dev)
        if b.sightline == 'global' or self.Nl == 1:
            nat.bin_reduce(b.grid, F64, nat.PB_RED_CROSS, a, sna, 1, self.k_bins, self._ells(self.Nl), scale, out,
                           b.ws)
            return out.cpu().numpy()
        # local sightline (pspec.py:522-544): multipole l crosses sum_m Y_lm(k) FT[Y_lm(r) a(r)]
        # (times -i for odd l)
        Nk = self.Nk
        nat.bin_reduce(b.grid, F64, nat.PB_RED_CROSS, a, sna, 1, self.k_bins, [(0, 0)], scale, out[:Nk], b.ws)
        a_real = b.to_real(a)
        for li in range(1, self.Nl):
            l = li * (2 - self.odd_l)
            lm = b.harmonics.apply_fourier(a_real, l)
            if l % 2:
                lm = lm * (-1j)
            nat.bin_reduce(b.grid, F64, nat.PB_RED_CROSS, lm, sna, 1, self.k_bins, [(0, 0)], scale,
                           out[li * Nk:(li + 1) * Nk], b.ws)
        return out.cpu().numpy()

    def _shot_inv_pa(self, PkA):
        """1/P_A on the grid, P_A interpolated with its end values beyond the table, 0 at
        k = 0 (pspec.py:505-508)."""
        from scipy.interpolate import interp1d
        b = self.base
        PA = interp1d(PkA[0], PkA[1], bounds_error=False, fill_value=(PkA[1][0], PkA[1][-1]))(b.modk_grid)
        inv = np.zeros_like(PA)
        nz = b.modk_grid != 0
        inv[nz] = 1. / PA[nz]
        return inv

    def _reference_field(self, seed):
        b = self.base
        re, im = b.reference_noise(seed + int(1e7))
        return b.grf_from_noise(torch.as_tensor(re, device=b.device)[None], torch.as_tensor(im, device=b.device)[None])

    def compute_covariance_contribution(self, seed, Pk_cov, verb=False):
        """Contribution of one GRF to the Gaussian covariance of the unwindowed estimator
        (pspec.py:149-162): the Fisher rows with S^-1 P replaced by S^-1 [P xi P^dag + N] S^-dag,
        xi the correlation of Pk_cov = [k, P0(, P2(, P4))] (no shot noise) and N the shot
        mask (the mask mean for a constant mask).  Same noise as compute_fisher_contribution."""
        if not self.const_mask:
            assert hasattr(self, 'mask_shot'), "Must supply mask_shot to compute shot-noise contribution"
        assert len(Pk_cov) != 0, "Must provide fiducial power spectrum if computing covariance!"
        assert len(np.asarray(Pk_cov).shape) == 2, "Pk should contain k and P_0, (and optionally P_2, P_4) columns"
        assert len(Pk_cov) in [2, 3, 4], "Pk should contain k and P_0, (and optionally P_2, P_4) columns"
        assert (len(Pk_cov) - 2) * 2 <= self.lmax, "Can't use higher multipoles than lmax"
        xi = self._xi_grids(np.asarray(Pk_cov, dtype=np.float64))
        return self._fisher_from_fields(self._reference_field(seed), xi=xi)[0].cpu().numpy()

    def compute_theory_contribution(self, seed, k_bins_theory, lmax_theory=None, include_wideangle=False,
                                    verb=False):
        """Fisher contribution and rectangular binning matrix of one GRF (pspec.py:164-196):
        row b of the binning matrix holds the cross spectra of the Fisher Q-map of bin b with
        A^-1 a in the theory k-bins, weighted by L_l(mu) (global) or with the harmonic
        transform sum_m Y_lm(k) FT[Y_lm(r) A^-1 a] (local), for l = 0, 2, .. lmax_theory (every
        l with odd_l).  include_wideangle (local, even l): the odd-l transforms of
        A^-1 a / |r| add the wide-angle terms to the l = 2, 4 blocks.
        Returns (fisher, binning_matrix)."""
        b = self.base
        k_bins_theory = np.asarray(k_bins_theory)
        assert np.max(k_bins_theory) < np.min(b.kNy), "k_max must be less than k_Nyquist!"
        assert np.min(k_bins_theory) >= np.max(b.kF), "k_min must be at least the k_fundamental!"
        assert np.max(k_bins_theory) <= b.Pfid[0][-1], "Fiducial power spectrum should extend up to k_max!"
        assert np.min(k_bins_theory) >= b.Pfid[0][0], "Fiducial power spectrum should extend down to k_min!"
        if lmax_theory is None:
            lmax_theory = self.lmax
        if include_wideangle:
            assert not b.sightline == 'global', "Wide-angle effects require local lines-of-sight!"
            assert not self.odd_l, "Cannot include wide-angle effects for odd l!"
            assert lmax_theory > 1, "There are no wide-angle effects for the monopole!"
            assert lmax_theory <= 4, "Higher-order effects not yet implemented!"
        elif not self.odd_l:
            assert lmax_theory % 2 == 0, "Must use even lmax if not including wide-angle effects!"
        if lmax_theory > 4:
            raise NotImplementedError("backend='cuda' implements theory multipoles up to l = 4")
        if b.sightline == 'local':
            assert lmax_theory >= self.lmax, "Can't use larger lmax for data than for theory!"
        if not np.all(np.diff(k_bins_theory) > 0):
            raise ValueError("k_bins_theory must be strictly increasing")
        odd_t = True if include_wideangle else bool(self.odd_l)
        nl_th = lmax_theory + 1 if (odd_t and not include_wideangle) else lmax_theory // 2 + 1   # pspec.py:218-228
        fish, bm = self._fisher_from_fields(self._reference_field(seed),
                                            theory=(k_bins_theory.astype(np.float64), nl_th, lmax_theory,
                                                    bool(include_wideangle), odd_t))
        return fish[0].cpu().numpy(), bm[0].cpu().numpy()
