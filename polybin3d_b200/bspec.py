"""Bispectrum estimators, backend='cuda' (mirrors PolyBin3D/bspec.py, global sightline).

Numerator: one r2c, one filter launch writing all Nl x Nk bin-filtered half spectra
(Theta_b L_l invP / W fused), one batched c2r, and the triplet contraction
sum_x g_b1 g_b2 g_l,b3 for every bin triplet (pb_triplet_contract).  Ideal Fisher and
symmetry factors reuse the same contraction on the binning functions (FP64).  The Monte
Carlo Fisher builds every Q-map leg with batched pair products, batched FFTs and three
accumulating filter launches, then forms Fisher rows per k-shell (pb_shell_rows), FP64.
"""
import numpy as np
import torch
from scipy.interpolate import interp1d

from . import _native as nat
from . import covariance
from . import pointing
from . import autotune
from . import realisations
from .harmonics import real_harmonics


class BSpec:
    """Bispectrum estimators (bspec.py:12-30 for the inputs).  Keyword-only addition:
    - contraction: 'auto' (tensor cores in precision='mixed' when built, else CUDA cores),
      'tc' or 'simt'.
    - dealias: synthesise the bin-filtered maps on the smallest FFT-friendly grid M with
      M > 3 K per axis (K = largest binned frequency index); every product of three such
      maps is then alias-free and sum_x over the M-grid equals (M/N)^3 times the sum over
      the full grid exactly, so results are unchanged up to rounding.  Default True.
    - synthesis: how bin-filtered maps are made: 'pruned' (pb_shell_synth: filter and
      inverse transform in one band-limited pass), 'cufft' (filter, then a cuFFT C2R of the
      whole grid) or 'auto' (pruned where the band limits allow it)."""

    def __init__(self, base, k_bins, lmax=0, mask=None, applySinv=None, k_bins_squeeze=None,
                 include_partial_triangles=False, add_GIC=False, mask_IC=None, add_RIC=False, radial_bins_RIC=[],
                 Pk_fid=None, mask_shot=None, applySinv_transpose=None, *, contraction='auto', dealias=True,
                 synthesis='auto', data_fft='fp64', verb=True):
        assert data_fft in ('fp64', 'fp32'), "data_fft must be 'fp64' or 'fp32'"
        self.data_fft = data_fft
        self.base = base
        self.applySinv = applySinv
        self.k_bins = np.asarray(k_bins)
        self.lmax = lmax
        self.Nk = len(k_bins) - 1
        self.Nl = self.lmax // 2 + 1
        self.include_partial_triangles = include_partial_triangles
        self.add_GIC = add_GIC
        self.add_RIC = add_RIC
        self.Pk_fid = Pk_fid
        self.applySinv_transpose = applySinv_transpose
        if contraction not in ('auto', 'tc', 'simt'):
            raise ValueError("contraction must be 'auto', 'tc' or 'simt'")
        self.contraction = contraction
        if synthesis not in ('auto', 'pruned', 'cufft'):
            raise ValueError("synthesis must be 'auto', 'pruned' or 'cufft'")
        self.synthesis = synthesis
        self._synth_ok = {}
        self.verb = verb

        if verb:
            print("")
        assert self.lmax % 2 == 0, "l-max must be even!"
        assert np.max(self.k_bins) < np.min(base.kNy), "k_max must be less than k_Nyquist!"
        assert np.min(self.k_bins) >= np.max(base.kF), "k_min must be at least the k_fundamental!"
        assert np.max(self.k_bins) <= base.Pfid[0][-1], "Fiducial power spectrum should extend up to k_max!"
        assert np.min(self.k_bins) >= base.Pfid[0][0], "Fiducial power spectrum should extend down to k_min!"
        if verb:
            print("Binning: %d bins in [%.3f, %.3f] h/Mpc" % (self.Nk, np.min(self.k_bins), np.max(self.k_bins)))

        # squeezed binning (bspec.py:53-65)
        if type(k_bins_squeeze) != type(None):
            self.k_bins_squeeze = np.asarray(k_bins_squeeze)
            self.Nk_squeeze = len(k_bins_squeeze) - 1
            assert (self.k_bins_squeeze[:self.Nk + 1] == self.k_bins).all(), "k_bins_squeeze must contain all non-squeezed bins!"
            assert np.max(self.k_bins_squeeze) < np.min(base.kNy), "k_max must be less than k_Nyquist!"
            assert np.min(self.k_bins_squeeze) >= np.max(base.kF), "k_min must be at least the k_fundamental!"
            assert np.max(self.k_bins_squeeze) <= base.Pfid[0][-1], "Fiducial power spectrum should extend up to k_max!"
            assert np.min(self.k_bins_squeeze) >= base.Pfid[0][0], "Fiducial power spectrum should extend down to k_min!"
            if verb:
                print("Squezed binning: %d bins in [%.3f, %.3f] h/Mpc" % (self.Nk_squeeze, np.min(self.k_bins_squeeze),
                                                                          np.max(self.k_bins_squeeze)))
        else:
            self.k_bins_squeeze = self.k_bins.copy()
            self.Nk_squeeze = self.Nk
        if not np.all(np.diff(self.k_bins_squeeze) > 0):
            raise ValueError("k_bins must be strictly increasing")

        # triangle bins (bspec.py:67-79)
        all_bins = []
        for l in range(0, self.lmax + 1, 2):
            for bin1 in range(self.Nk):
                for bin2 in range(bin1, self.Nk_squeeze):
                    for bin3 in range(bin2, self.Nk_squeeze):
                        if not self._check_bin(bin1, bin2, bin3):
                            continue
                        all_bins.append((bin1, bin2, bin3, l))
        self.all_bins = np.asarray(all_bins, dtype=np.int64)
        self.N_bins = len(self.all_bins)
        self.N3 = self.N_bins // self.Nl
        if verb:
            print("l-max: %d" % (self.lmax))
            print("N_bins: %d" % self.N_bins)
        assert type(self.lmax) == int, "l-max must be an integer!"
        assert self.lmax <= 4, "Only l-max<=4 is currently supported!"

        # mask (bspec.py:86-110)
        if type(mask) == type(None):
            self.const_mask = True
            self.mask_mean = 1.
            self.cube_mask_mean = 1.
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
            self.cube_mask_mean = np.mean(self.mask ** 3)
        if verb:
            print("Mask: constant" if self.const_mask else "Mask: spatially varying")
        if type(mask_shot) != type(None):
            self.mask_shot = mask_shot.astype(np.float64)

        # S^-1 (bspec.py:117-124): the trivial filter, or the caller's, applied to device maps;
        # its transpose (used by the covariance) defaults to itself
        self._custom_sinv = self.applySinv is not None
        if self._custom_sinv and type(self.applySinv_transpose) != type(lambda x: x):
            self.applySinv_transpose = self.applySinv
            if verb:
                print("## Caution: assuming S^-1 is Hermitian!")
        # integral constraints (bspec.py:126-136)
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

        # fiducial weighting 1/P_fid (bspec.py:138-156); None -> unit weight on every binned mode
        self._unit_w = (type(self.Pk_fid) != str and (np.asarray(self.Pk_fid) == None).all()) or \
                       (isinstance(self.Pk_fid, str) and self.Pk_fid == 'default' and base._unit_pk)  # noqa: E711
        if not (isinstance(self.Pk_fid, str) and self.Pk_fid == 'default') and not self._unit_w:
            assert len(self.Pk_fid) == 2, "Pk should contain k and P_0(k) columns"
        self._plans = {}
        self._set_idx = {}
        self._captured = None
        self._shell_modes = None
        self.map_grid = self._dealiased_grid() if dealias else tuple(int(n) for n in base.gridsize)

    def _ylm(self, kind):
        """Real harmonics of positions ('r') or wavevectors ('k') by even l, as the
        reference's Ylm_real / Ylm_fourier (bspec.py:158-169): FP64 device grids, made on
        first use; None unless the sightline is local and lmax > 0."""
        if self.base.sightline != 'local' or self.lmax == 0:
            return None
        return {l: self.base.harmonics._grid(kind, l, torch.float64) for l in range(2, self.lmax + 1, 2)}

    @property
    def Ylm_real(self):
        return self._ylm('r')

    @property
    def Ylm_fourier(self):
        return self._ylm('k')

    # ------------------------------------------------------------------------------
    # binning helpers (bspec.py:171-220)
    # ------------------------------------------------------------------------------
    def _check_bin(self, bin1, bin2, bin3):
        """Triangle condition on bin centres, or on edges for partial triangles (bspec.py:171-199)."""
        if self.include_partial_triangles:
            k3_hi = self.k_bins_squeeze[bin1 + 1] + self.k_bins_squeeze[bin2 + 1]
            if bin1 > bin2:
                k3_lo = self.k_bins_squeeze[bin1] - self.k_bins_squeeze[bin2 + 1]
            elif bin1 == bin2:
                k3_lo = 0.
            else:
                k3_lo = self.k_bins_squeeze[bin2] - self.k_bins_squeeze[bin1 + 1]
            if self.k_bins_squeeze[bin3] >= k3_hi - 1e-10 or self.k_bins_squeeze[bin3 + 1] <= k3_lo + 1e-10:
                return 0
            return 1
        k1 = 0.5 * (self.k_bins[bin1] + self.k_bins[bin1 + 1])
        k2 = 0.5 * (self.k_bins_squeeze[bin2] + self.k_bins_squeeze[bin2 + 1])
        k3 = 0.5 * (self.k_bins_squeeze[bin3] + self.k_bins_squeeze[bin3 + 1])
        if k3 < abs(k1 - k2) or k3 > k1 + k2:
            return 0
        return 1

    def get_ks(self):
        """Central k1, k2, k3 of every triangle bin (bspec.py:201-220)."""
        k1s, k2s, k3s = [], [], []
        for bin1 in range(self.Nk):
            k1 = 0.5 * (self.k_bins[bin1] + self.k_bins[bin1 + 1])
            for bin2 in range(bin1, self.Nk_squeeze):
                k2 = 0.5 * (self.k_bins_squeeze[bin2] + self.k_bins_squeeze[bin2 + 1])
                for bin3 in range(bin2, self.Nk_squeeze):
                    k3 = 0.5 * (self.k_bins_squeeze[bin3] + self.k_bins_squeeze[bin3 + 1])
                    if not self._check_bin(bin1, bin2, bin3):
                        continue
                    k1s.append(k1)
                    k2s.append(k2)
                    k3s.append(k3)
        return np.asarray([k1s, k2s, k3s])

    def _dealiased_grid(self):
        """Per axis, the smallest even 2^a 3^b 5^c size M > 3 K (K = floor(k_max / kF)) not
        above the data grid (the lengths the pruned synthesis transforms)."""
        b = self.base
        kmax = float(np.max(self.k_bins_squeeze))
        dims = []
        for i in range(3):
            K = int(np.floor(kmax / b.kF[i]))
            m = 3 * K + 1
            while True:
                r = m
                for f in (2, 3, 5):
                    while r % f == 0:
                        r //= f
                if r == 1 and m % 2 == 0:
                    break
                m += 1
            dims.append(int(min(m, int(b.gridsize[i]))))
        return tuple(dims)

    @property
    def map_scale(self):
        """(N/M)^3: converts a sum over the map grid into the sum over the data grid."""
        return float(np.prod(self.base.gridsize) / np.prod(self.map_grid))

    # ------------------------------------------------------------------------------
    # device helpers
    # ------------------------------------------------------------------------------
    @property
    def invPk0(self):
        """1/P_fid on the half grid (bspec.py:139-156), host FP64."""
        b = self.base
        if isinstance(self.Pk_fid, str) and self.Pk_fid == 'default':
            return b.invPk0_grid
        if self._unit_w:
            k_tmp = np.arange(np.min(b.kF) / 10., np.max(b.kNy) * 2, np.min(b.kF) / 10.)
            Pfid = np.asarray([k_tmp, 1. + 0. * k_tmp])
        else:
            Pfid = np.asarray(self.Pk_fid)
        P = interp1d(Pfid[0], Pfid[1], bounds_error=False, fill_value=0.)(b.modk_grid)
        inv = np.zeros(P.shape, dtype=np.float64)
        inv[P != 0] = 1. / P[P != 0]
        return inv

    def _invp_device(self):
        """Device 1/P_fid weight, or None when it is 1 on every binned mode."""
        if self._unit_w:
            return None
        return self.base.to_device_grid(('bk_invp', id(self)), lambda: self.invPk0, torch.float64)

    def _data_weight(self, dtype):
        """invP / W on the half grid for the ideal numerator (None when identically 1 on the
        binned modes).  With unit weighting invP is 1 on every binned mode, so the global
        sightline skips it; the local sightline's l > 0 maps mix all modes of the weighted
        field (through the real-space harmonics), so there invP keeps its zero at k = 0."""
        b = self.base
        unit = self._unit_w and not (b.sightline == 'local' and self.lmax > 0)
        if unit and b.pixel_window == 'none':
            return None

        def f():
            w = np.ones(b.nhalf_shape) if unit else self.invPk0.copy()
            if b.pixel_window != 'none':
                W = b.pixel_window_grid
                nz = W != 0
                w = np.where(nz, w / np.where(nz, W, 1.), 0.)
            return w
        return b.to_device_grid(('bk_dataw', id(self)), f, dtype)

    def _plan(self, key, n_a, n_b, n_c, idx):
        if key is None:
            return nat.TripletPlan(n_a, n_b, n_c, idx, self.base.device)
        key = (key, n_a, n_b, n_c)
        p = self._plans.get(key)
        if p is None:
            p = nat.TripletPlan(n_a, n_b, n_c, idx, self.base.device)
            self._plans[key] = p
        return p

    def _method(self, dtype):
        if dtype == torch.float64 or self.contraction == 'simt':
            return nat.PB_TRIPLET_SIMT
        if self.contraction == 'tc':
            return nat.PB_TRIPLET_TC
        return nat.PB_TRIPLET_TC if tc_available() else nat.PB_TRIPLET_SIMT

    def _contract(self, key, A, B, C, idx, scale=1.0):
        """FP64 triplet sums of maps A, B, C; maps on the dealiased grid are rescaled to
        full-grid sums."""
        b = self.base
        plan = self._plan(key, A.shape[0], B.shape[0], C.shape[0], idx)
        out = torch.empty(plan.n_trip, dtype=torch.float64, device=b.device)
        if tuple(A.shape[1:]) != tuple(int(n) for n in b.gridsize):
            scale = scale * float(np.prod(b.gridsize)) / float(np.prod(A.shape[1:]))
        method = self._method(A.dtype)
        if method == nat.PB_TRIPLET_TC and getattr(plan, "tc_unsupported", False):
            method = nat.PB_TRIPLET_SIMT
        try:
            autotune.contract(plan, A, B, C, out, b.ws, method, scale)
        except NotImplementedError:
            # the tensor-core tiling does not fit this shape (too many pair rows or maps
            # for shared memory / TMEM): the CUDA-core kernel takes it
            if method != nat.PB_TRIPLET_TC or self.contraction == 'tc':
                raise
            plan.tc_unsupported = True
            plan.contract(A, B, C, out, b.ws, method=nat.PB_TRIPLET_SIMT, scale=scale)
        return out

    def _binned_maps(self, src, specs, w, dtype, coarse=True, out=None):
        """Real maps irfftn(Theta_b L_l1 L_l2 * w^wp * src) for specs [(b, l1, l2, scale)], batched.
        coarse: synthesise them on the dealiased map grid (same 1/N^3 normalisation).
        out: optional contiguous (len(specs), *grid) tensor to write them into."""
        b = self.base
        ks = self.k_bins_squeeze
        cd = torch.complex128 if dtype == torch.float64 else torch.complex64
        prec = nat.precision_of(dtype)
        # FP32 maps from an FP64 spectrum: the pruned synthesis reads it as it is
        src64 = src is not None and src.dtype == torch.complex128 and dtype == torch.float32
        sprec = nat.PB_F32_SRC_F64 if src64 else prec
        dims = self.map_grid if coarse else tuple(int(n) for n in b.gridsize)
        wp = 0 if w is None else 1
        # spec: (bin, l1, l2, scale[, source index]); the sources lie src_stride apart
        maps = [(sp[4] if len(sp) > 4 else 0, ks[sp[0]], ks[sp[0] + 1], sp[1], sp[2], sp[3] / b.nreal, wp)
                for sp in specs]
        if isinstance(out, nat.TiledMaps):
            # a tiled set comes from the pruned synthesis only (one pass)
            if self.synthesis == 'cufft' or not self._synth_ok.get(dims, True):
                raise NotImplementedError("tiled maps need the pruned synthesis")
            nat.shell_synth(b.grid, sprec, src, out, maps, dims, b.ws, w=w, src_stride=b.nhalf)
            b.n_FFTs_reverse += len(specs)
            return out
        if self.synthesis != 'cufft' and self._synth_ok.get(dims, True):
            if out is None:
                out = torch.empty((len(specs),) + tuple(dims), dtype=dtype, device=b.device)
            try:
                nat.shell_synth(b.grid, sprec, src, out, maps, dims, b.ws, w=w, src_stride=b.nhalf)
                b.n_FFTs_reverse += len(specs)
                return out
            except NotImplementedError:
                if self.synthesis == 'pruned':
                    raise
                self._synth_ok[dims] = False
        if src64:
            src = src.to(cd)
        hs = (dims[0], dims[1], dims[2] // 2 + 1)
        half = torch.empty((len(specs),) + hs, dtype=cd, device=b.device)
        nat.spectral_filter(b.grid, prec, src, half, maps, w=w, src_stride=b.nhalf,
                            out_n=None if coarse is False or dims == tuple(int(n) for n in b.gridsize) else dims)
        b.n_FFTs_reverse += len(specs)
        return b.fft_c2r(half, out=out)

    # ------------------------------------------------------------------------------
    # symmetry factors (bspec.py:222-279)
    # ------------------------------------------------------------------------------
    def _compute_symmetry_factor(self):
        if self.verb:
            print("Computing degeneracy factor")
        sym = []
        for (b1, b2, b3, l) in self.all_bins[:self.N3]:
            if b1 == b2 and b1 == b3:
                sym.append(6.)
            elif b1 == b2 or b1 == b3 or b2 == b3:
                sym.append(2.)
            else:
                sym.append(1.)
        if self.lmax > 0:
            b = self.base
            nks = self.Nk_squeeze
            w = self._invp_device()
            bins = self._binned_maps(None, [(i, 0, 0, 1.0) for i in range(nks)], w, torch.float64)
            kg = b.k_grids
            invP = np.ones(b.nhalf_shape) if self._unit_w else self.invPk0
            for l in range(2, self.lmax + 1, 2):
                rows = self.all_bins[self.all_bins[:, 3] == l]
                need = sorted({int(r[2]) for r in rows if (r[0] != r[1] and r[1] == r[2]) or (r[0] == r[1] == r[2])})
                # sum over m of bins-weighted squares of the Y_lm-weighted binning functions
                pair_idx = sorted({(int(r[0]), int(r[2])) for r in rows if r[0] != r[1] and r[1] == r[2]} |
                                  {(int(r[2]), int(r[2])) for r in rows if r[0] == r[1] == r[2]})
                num = {p: 0.0 for p in pair_idx}
                if pair_idx:
                    for y in real_harmonics(kg, l):
                        wy = torch.as_tensor(invP * y, device=b.device)
                        ym = self._binned_maps(None, [(i, 0, 0, 1.0) for i in need], wy, torch.float64)
                        pos = {bb: i for i, bb in enumerate(need)}
                        idx = np.asarray([(p[0], pos[p[1]], pos[p[1]]) for p in pair_idx], dtype=np.int32)
                        vals = self._contract(None, bins, ym, ym, idx).cpu().numpy()
                        for p, v in zip(pair_idx, vals):
                            num[p] += v
                    idx3 = np.asarray([(p[0], p[1], p[1]) for p in pair_idx], dtype=np.int32)
                    den = dict(zip(pair_idx, self._contract(('sym_den', l), bins, bins, bins, idx3).cpu().numpy()))
                for (b1, b2, b3, ll) in rows:
                    if b1 != b2 and b2 != b3:
                        sym.append(1.)
                    elif b1 == b2 and b2 != b3:
                        sym.append(2.)
                    elif b1 != b2 and b2 == b3:
                        sym.append(1. + num[(b1, b3)] / den[(b1, b3)])
                    else:
                        sym.append(2. * (1. + 2. * num[(b3, b3)] / den[(b3, b3)]))
        self.sym_factor = np.asarray(sym)
        assert len(self.sym_factor) == self.N_bins

    # ------------------------------------------------------------------------------
    # numerator (bspec.py:895-983)
    # ------------------------------------------------------------------------------
    def _triplet_index(self):
        ab = self.all_bins
        return np.stack([ab[:, 0], ab[:, 1], (ab[:, 3] // 2) * self.Nk_squeeze + ab[:, 2]], axis=1).astype(np.int32)

    def _g_maps(self, xk, w, scale, out=None, rd=None):
        """All Nl x Nk_squeeze bin-filtered maps g[l/2, b] of one weighted spectrum, as real
        maps of dtype rd (default: the spectrum's; FP32 maps may come from an FP64 spectrum)."""
        rd = rd or xk.real.dtype
        if self.base.sightline == 'local' and self.lmax > 0:
            if xk.real.dtype != rd:
                xk = xk.to(torch.complex64 if rd == torch.float32 else torch.complex128)
            return self._g_maps_local(xk, w, scale, out)
        specs = [(bb, l, 0, scale) for l in range(0, self.lmax + 1, 2) for bb in range(self.Nk_squeeze)]
        return self._binned_maps(xk, specs, w, rd, out=out)

    def _g_maps_local(self, xk, w, scale, out=None, coarse=True):
        """Local sightline (bspec.py:932-954): with D = scale w xk and d = irfftn(D), the
        l = 0 maps filter D and the l > 0 maps filter sum_m Y_lm(k) FT[Y_lm(r) d(r)], all with
        the plain bin filter, in one synthesis over the stacked sources."""
        b = self.base
        prec = nat.precision_of(xk.dtype)
        D = torch.empty_like(xk)
        nat.spectral_filter(b.grid, prec, xk.contiguous(), D,
                            [(0, -1.0, np.inf, 0, 0, float(scale), 0 if w is None else 1)], w=w)
        d = b.to_real(D)
        srcs = torch.stack([D] + [b.harmonics.apply_fourier(d, l) for l in range(2, self.lmax + 1, 2)])
        specs = [(bb, 0, 0, 1.0, l // 2) for l in range(0, self.lmax + 1, 2) for bb in range(self.Nk_squeeze)]
        return self._binned_maps(srcs, specs, None, xk.real.dtype, coarse=coarse, out=out)

    def _compute_bk_numerator(self, data, include_linear_term=True, filtering='ideal', verb=False):
        assert filtering in ['ideal', 'Sinv'], "Unknown filtering option supplied!"
        if (not hasattr(self, 'preload')) and include_linear_term:
            raise Exception("Need to generate or specify bias simulations!")
        b = self.base
        if not isinstance(data, torch.Tensor):
            assert type(data[0, 0, 0]) in [np.float32, np.float64], "Data must be of type float32 or float64!"
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        B3 = self._bk_cubic(data, filtering, linear=include_linear_term)
        norm = b.volume / float(b.gridsize.prod()) / self.sym_factor
        return B3.cpu().numpy() * norm

    def _data_spectrum(self, x, keep64=False):
        """rfftn of a data field.  With FP32 maps (precision='mixed') the transform itself runs
        in FP64 unless data_fft='fp32': the FP32 r2c's rounding (relative to the largest modes,
        so large on the weak high-k modes) is the biggest error of the mixed path on the bins
        whose triple products cancel (quadrupoles near zero); rounding the FP64 spectrum to
        FP32 afterwards costs ~1e-7 per mode.  keep64: return that FP64 spectrum as it is, for
        a caller whose synthesis reads it directly (FP32 maps, no rounded copy)."""
        b = self.base
        if x.dtype == torch.float32 and self.data_fft == 'fp64':
            b.n_FFTs_forward += 1
            xk = b.fft_r2c(nat.widen(x.contiguous()))
            return xk if keep64 else xk.to(torch.complex64)
        return b.to_fourier(x)

    def _bk_cubic(self, data, filtering, linear=False):
        """Device FP64 sums B3[i] (assemble_b3 of the g-maps), plus the linear term
        B1 = -1/N_it sum_ii assemble_b1(g, g_ii) of the bias simulations when `linear`
        (bspec.py:958-978)."""
        b = self.base
        x = b.as_device(data)
        xk = self._data_spectrum(x, keep64=filtering == 'ideal' and not linear)
        rd = x.dtype
        if filtering == 'ideal':
            w = self._data_weight(rd)
            scale = 1.0 / self.cube_mask_mean ** (1. / 3.)
        elif self._custom_sinv:                                          # bspec.py:912-929
            cd = torch.complex128 if rd == torch.float64 else torch.complex64
            xk = self._sinv_data(data).to(cd)
            w = None
            scale = 1.0
        else:
            w = None
            if b.pixel_window != 'none':
                w = b.to_device_grid(('bk_invwin', id(self)), lambda: self._inv_window(), rd)
            scale = 1.0
        if not linear:
            return self._b3_sums(xk, w, scale, rd)
        # data maps and one simulation's maps side by side: X = [g; g_ii]
        n = self.Nl * self.Nk_squeeze
        X = torch.empty((2 * n,) + tuple(self.map_grid), dtype=rd, device=b.device)
        G, S = X[:n], X[n:]
        self._g_maps(xk, w, scale, out=G)
        out = self._contract('b3', G, G, G, self._triplet_index())
        b1 = torch.zeros(self.N_bins, dtype=torch.float64, device=b.device)
        for ii in range(self.N_it):
            self._g_maps(self._sim_spectrum(ii, rd), None, 1.0, out=S)
            b1 += self._set_sums('b1', X, n, ((0, 1, 1), (1, 0, 1), (1, 1, 0)))
        return out - b1 / self.N_it

    def _b3_sums(self, xk, w, scale, rd=None):
        """FP64 sums B3[i] = assemble_b3 of the g-maps of one weighted spectrum.  With the
        tensor-core contraction there are two routes: the g-maps synthesised straight into a
        tiled set (the contraction's staging layout: each tile of voxels of all maps is one
        contiguous copy and the MMA operand comes pre-split), or plain maps staged by 2-D TMA
        boxes.  The faster for this shape (synthesis and contraction timed together) is found
        once and cached by the autotuner; the two agree to FP32 rounding.  rd: the maps' dtype
        (default: the spectrum's)."""
        rd = rd or xk.real.dtype
        if self._tiled_ok(rd) and self._b3_route(xk, w, scale, rd) == "tiled":
            out = self._b3_tiled(xk, w, scale, rd)
            if out is not None:
                return out
        return self._b3_plain(xk, w, scale, rd)

    def _b3_plain(self, xk, w, scale, rd=None):
        G = self._g_maps(xk, w, scale, rd=rd)
        return self._contract('b3', G, G, G, self._triplet_index())

    def _b3_tiled(self, xk, w, scale, rd=None):
        """The tiled route, or None when a tiled set cannot be made or contracted here."""
        T = self._g_maps_tiled(xk, w, scale, rd)
        if T is None:
            return None
        plan = self._plan('b3', T.n_maps, T.n_maps, T.n_maps, self._triplet_index())
        out = torch.empty(plan.n_trip, dtype=torch.float64, device=self.base.device)
        try:
            return autotune.contract_tiled(plan, T, out, self.base.ws, self._grid_scale(T.shape))
        except NotImplementedError:
            if self.contraction == 'tc':
                raise
            self._tiled = False
            return None

    def _b3_route(self, xk, w, scale, rd=None):
        b = self.base
        key = "b3route|%s|%s|%d|%d|%s" % (autotune.device_tag(b.device), ",".join(str(int(n)) for n in self.map_grid),
                                          self.Nl * self.Nk_squeeze, self.Nk_squeeze, b.sightline)
        def tiled():
            if self._b3_tiled(xk, w, scale, rd) is None:
                raise NotImplementedError("no tiled set for this shape")
        return autotune.tuner().choose_route(key, {"tiled": tiled, "plain": lambda: self._b3_plain(xk, w, scale, rd)})

    def _tiled_ok(self, dtype):
        return (getattr(self, '_tiled', True) and self.synthesis != 'cufft' and
                self._method(dtype) == nat.PB_TRIPLET_TC and self.Nl * self.Nk_squeeze <= 64)

    def _grid_scale(self, shape):
        """Factor taking sums over the (dealiased) map grid `shape` to full-grid sums."""
        b = self.base
        if tuple(shape) != tuple(int(n) for n in b.gridsize):
            return float(np.prod(b.gridsize)) / float(np.prod(shape))
        return 1.0

    def _g_maps_tiled(self, xk, w, scale, rd=None):
        """The g-maps of _g_maps as a tiled set, or None when the pruned synthesis cannot
        make them (the caller takes the plain path)."""
        b = self.base
        # the monopole maps (the first Nk_squeeze) are the pair factors of every triplet
        T = nat.TiledMaps(self.Nl * self.Nk_squeeze, self.Nk_squeeze, self.map_grid, b.device)
        try:
            self._g_maps(xk, w, scale, out=T, rd=rd or xk.real.dtype)
        except NotImplementedError:
            self._tiled = False
            return None
        return T

    def _set_sums(self, key, X, n, terms):
        """FP64 sum over `terms` (ta, tb, tc) of the triplet sums
        sum_x X_ta[0,b1](x) X_tb[0,b2](x) X_tc[l,b3](x), where X holds map sets of n maps each
        side by side (set t = X[t n:(t+1) n], maps ordered (l/2, b)).  Terms that share the
        C set go through one contraction with A = B = X and C = that set (rows of X, staged
        once); each pair is listed with its smaller map index first, since the products
        commute, so the pair rows of different terms are shared, and triplets that coincide
        (b1 = b2 in the two mixed orderings) are contracted once and gathered back."""
        t = self._triplet_index().astype(np.int64)
        i1, i2, i3 = t[:, 0], t[:, 1], t[:, 2]
        nb = self.N_bins
        by_c = {}
        for (ta, tb, tc) in terms:
            by_c.setdefault(tc, []).append((ta, tb))
        total = None
        for tc in sorted(by_c):
            ab = tuple(by_c[tc])
            ck = (key, tc, ab)
            hit = self._set_idx.get(ck)
            if hit is None:
                rows = []
                for (ta, tb) in ab:
                    p, q = ta * n + i1, tb * n + i2
                    rows.append(np.stack([np.minimum(p, q), np.maximum(p, q), i3], axis=1))
                uniq, inv = np.unique(np.concatenate(rows), axis=0, return_inverse=True)
                hit = (uniq.astype(np.int32), torch.as_tensor(inv.reshape(-1), device=self.base.device))
                self._set_idx[ck] = hit
            idx, inv = hit
            out = self._contract(ck, X, X, X[tc * n:(tc + 1) * n], idx)[inv].view(len(ab), nb).sum(0)
            total = out if total is None else total + out
        return total

    # ------------------------------------------------------------------------------
    # bias simulations for the linear term (bspec.py:281-410)
    # ------------------------------------------------------------------------------
    def _sim_spectrum(self, ii, dtype):
        """The Fourier map of bias simulation ii, pixel window divided out, as the map dtype."""
        xs = self._sim_store[ii] if self.preload else self.load_sim_data(ii)
        cd = torch.complex128 if dtype == torch.float64 else torch.complex64
        return xs if xs.dtype == cd else xs.to(cd)

    def _process_sim(self, sim, input_type='real'):
        """_process_sim up to its g-maps (bspec.py:281-300): the Fourier map of one
        simulation with the pixel window divided out (trivial S^-1), stored in the base
        precision.  The g-maps are synthesised from it when the linear term is formed, so a
        simulation holds one half spectrum of device memory instead of Nl x Nk maps."""
        b = self.base
        if self._custom_sinv:
            return self._sinv_data(sim, input_type).to(b.complex_dtype)
        if input_type == 'real':
            xk = b.to_fourier(b.as_device(sim))
        else:
            xk = torch.as_tensor(sim, device=b.device).to(b.complex_dtype).contiguous()
        if b.pixel_window != 'none':
            prec = nat.precision_of(xk.dtype)
            rd = torch.float64 if prec == nat.PB_F64 else torch.float32
            w = b.to_device_grid(('bk_invwin', id(self)), lambda: self._inv_window(), rd)
            out = torch.empty_like(xk)
            nat.spectral_filter(b.grid, prec, xk, out, [(0, -1.0, np.inf, 0, 0, 1.0, 1)], w=w)
            xk = out
        return xk

    def _generated_sim(self, ii, Pk_input):
        """load_sim_data of generate_sims (bspec.py:377-392): the GRF of seed 1e5 + ii
        (the reference's own noise draw), times the mask mean (constant mask) or through the
        mask in real space, in FP64.  The pixel window that the reference multiplies in and
        _process_sim divides out again is left out of both steps."""
        b = self.base
        re, im = b.reference_noise(int(1e5) + ii)
        nre = torch.as_tensor(re, device=b.device)
        nim = torch.as_tensor(im, device=b.device)
        a = b.grf_from_noise(nre, nim, Pk_input if len(Pk_input) else None, include_pixel_window=False)
        F64 = nat.PB_F64
        if self.const_mask:
            out = torch.empty_like(a)
            nat.spectral_filter(b.grid, F64, a, out, [(0, -1.0, np.inf, 0, 0, float(self.mask_mean), 0)])
            if self._custom_sinv:
                out = self._sinv(out, 'fourier', 'fourier')
            return out.to(b.complex_dtype)
        s = b.to_real(a)
        self._pointing()(s, False, out=s)
        if self._custom_sinv:
            y = self._sinv(b.to_fourier(s), 'fourier', 'fourier') if b.pixel_window != 'none' else \
                self._sinv(s, 'real', 'fourier')
            return y.to(b.complex_dtype)
        return b.to_fourier(s).to(b.complex_dtype)

    def _inv_window(self):
        W = self.base.pixel_window_grid
        nz = W != 0
        return np.where(nz, 1. / np.where(nz, W, 1.), 0.)

    def _sinv(self, x, input_type, output_type, transpose=False):
        """The caller's S^-1 (or S^-dag) on one device map; the result as a contiguous FP64
        device tensor (half spectrum or real map)."""
        f = self.applySinv_transpose if transpose else self.applySinv
        y = f(x, input_type=input_type, output_type=output_type)
        if not isinstance(y, torch.Tensor):
            y = torch.as_tensor(np.ascontiguousarray(y))
        dt = torch.complex128 if output_type == 'fourier' else torch.float64
        return y.to(device=self.base.device, dtype=dt).contiguous()

    def _sinv_data(self, data, input_type='real'):
        """S^-1 of data or of a simulation in Fourier space with the caller's S^-1, the pixel
        window divided out first when there is one (bspec.py:287-300, 733-742, 912-929)."""
        b = self.base
        if b.pixel_window == 'none':
            x = b.as_device(data, torch.float64) if input_type == 'real' else data
            return self._sinv(x, input_type, 'fourier')
        if input_type == 'real':
            xk = b.to_fourier(b.as_device(data, torch.float64))
        else:
            xk = torch.as_tensor(data, device=b.device).to(torch.complex128).contiguous().clone()
        w = b.to_device_grid(('bk_invwin', id(self)), lambda: self._inv_window(), torch.float64)
        nat.spectral_filter(b.grid, nat.PB_F64, xk, xk, [(0, -1.0, np.inf, 0, 0, 1.0, 1)], w=w)
        return self._sinv(xk, 'fourier', 'fourier')

    def Bk_numerator(self, data, include_linear_term=True, verb=False):
        """Numerator of the unwindowed estimator (bspec.py:429-439); the linear term needs
        bias simulations (generate_sims or load_sims)."""
        if not self.const_mask:
            assert data.shape == self.mask.shape, "Data must have same shape as the mask!"
        return self._compute_bk_numerator(data, include_linear_term=include_linear_term, filtering='Sinv', verb=verb)

    def Bk_numerator_ideal(self, data, verb=False):
        """Numerator of the ideal estimator (bspec.py:986-997)."""
        if not self.const_mask:
            assert data.shape == self.mask.shape, "Data must have same shape as the mask!"
        return self._compute_bk_numerator(data, include_linear_term=False, filtering='ideal', verb=verb)

    def load_sims(self, load_sim, N_sims, verb=False, input_type='real', preload=True):
        """Bias simulations for the linear term from a loader load_sim(ii), real- or
        Fourier-space (bspec.py:324-352).  preload=True keeps each simulation's filtered
        Fourier map on the device; preload=False calls the loader again every time."""
        self.N_it = N_sims
        print("Using %d Monte Carlo simulations" % self.N_it)
        if preload:
            self.preload = True
            self._sim_store = []
            for ii in range(self.N_it):
                if verb: print("Loading bias simulation %d of %d" % (ii + 1, self.N_it))
                self._sim_store.append(self._process_sim(load_sim(ii), input_type=input_type))
        else:
            self.preload = False
            if verb: print("No preloading; simulations will be loaded and accessed at runtime.")
            self.load_sim_data = lambda ii: self._process_sim(load_sim(ii), input_type=input_type)

    def generate_sims(self, N_sim, Pk_input=[], verb=False, preload=True):
        """N_sim Gaussian bias simulations of the fiducial (or given) spectrum through the
        mask, seeds 1e5 + ii (bspec.py:354-410)."""
        self.N_it = N_sim
        print("Using %d Monte Carlo simulations" % self.N_it)
        if preload:
            self.preload = True
            self._sim_store = []
            for ii in range(self.N_it):
                if verb: print("Generating bias simulation %d of %d" % (ii + 1, self.N_it))
                self._sim_store.append(self._generated_sim(ii, Pk_input))
        else:
            self.preload = False
            if verb: print("No preloading; simulations will be loaded and accessed at runtime.")
            self.load_sim_data = lambda ii: self._generated_sim(ii, Pk_input)

    # ------------------------------------------------------------------------------
    # ideal Fisher (bspec.py:999-1083)
    # ------------------------------------------------------------------------------
    def compute_fisher_ideal(self, discreteness_correction=True, verb=False):
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        if self.verb:
            print("Computing ideal Fisher matrix")
        nks = self.Nk_squeeze
        w = self._invp_device()
        idx3 = self.all_bins[:self.N3, :3].astype(np.int32)
        b = self.base
        if discreteness_correction:
            fish = np.zeros((self.N_bins, self.N_bins))
            u = self._binned_maps(None, [(bb, l, 0, 1.0) for l in range(0, self.lmax + 1, 2) for bb in range(nks)], w,
                                  torch.float64)
            u0 = u[:nks]
            for l in range(0, self.lmax + 1, 2):
                for lp in range(l, self.lmax + 1, 2):
                    ull = self._binned_maps(None, [(bb, l, lp, 1.0) for bb in range(nks)], w, torch.float64)
                    T1 = self._contract('fid', u0, u0, ull, idx3).cpu().numpy()
                    T2 = self._contract('fid', u0, u[l // 2 * nks:(l // 2 + 1) * nks],
                                        u[lp // 2 * nks:(lp // 2 + 1) * nks], idx3).cpu().numpy()
                    for i in range(self.N3):
                        b1, b2, b3 = idx3[i]
                        if b1 != b2 and b2 != b3:
                            v = T1[i]
                        elif b1 == b2 and b2 != b3:
                            v = 2. * T1[i]
                        elif b1 != b2 and b2 == b3:
                            v = T2[i] + T1[i]
                        else:
                            v = 4. * T2[i] + 2. * T1[i]
                        fish[l // 2 * self.N3 + i, lp // 2 * self.N3 + i] = v
            fish = fish + fish.T - np.diag(np.diag(fish))
            scaling = b.gridsize.prod() ** 2 / b.volume
            fish = fish / np.outer(self.sym_factor, self.sym_factor) * scaling
        else:
            u0 = self._binned_maps(None, [(bb, 0, 0, 1.0) for bb in range(nks)], w, torch.float64)
            N_triangles = self._contract('fid', u0, u0, u0, idx3).cpu().numpy()
            fish_diag = np.zeros(self.N_bins)
            for l in range(0, self.lmax + 1, 2):
                fish_diag[l // 2 * self.N3:(l // 2 + 1) * self.N3] = N_triangles / (2. * l + 1.)
            fish = np.diag(fish_diag / self.sym_factor) * b.gridsize.prod() ** 2 / b.volume
        self.fish_ideal = fish
        self.inv_fish_ideal = np.linalg.inv(self.fish_ideal)
        self.discreteness_correction = discreteness_correction
        return fish

    def Bk_ideal(self, data, fish_ideal=[], discreteness_correction=True, verb=False):
        """Ideal estimator (bspec.py:1085-1118).  `data` may also be a list of fields: they
        are streamed (the host-to-device copy of field i+1 overlaps the estimator of field i,
        on its own stream, when the fields are pinned torch tensors) and a list of dicts is
        returned."""
        if len(fish_ideal) != 0:
            self.fish_ideal = fish_ideal
            self.inv_fish_ideal = np.linalg.inv(fish_ideal)
        if not hasattr(self, 'inv_fish_ideal'):
            self.compute_fisher_ideal(discreteness_correction=discreteness_correction, verb=verb)
        elif getattr(self, 'discreteness_correction', discreteness_correction) != discreteness_correction:
            self.compute_fisher_ideal(discreteness_correction=discreteness_correction, verb=verb)
        if isinstance(data, (list, tuple)):
            return [self._bk_dict(r) for r in self._bk_ideal_stream(data)]
        Bk_num_ideal = self.Bk_numerator_ideal(data, verb=verb)
        return self._bk_dict(np.matmul(self.inv_fish_ideal, Bk_num_ideal))

    def _bk_dict(self, Bk_out):
        Bk_dict = {}
        index = 0
        for l in range(0, self.lmax + 1, 2):
            Bk_dict['b%s' % l] = Bk_out[index:index + self.N3]
            index += self.N3
        return Bk_dict

    def _bk_ideal_stream(self, fields):
        """F^-1 B_num for each field; two device field buffers, copies on a side stream."""
        b = self.base
        for f in fields:
            if not isinstance(f, torch.Tensor):
                assert type(f[0, 0, 0]) in [np.float32, np.float64], "Data must be of type float32 or float64!"
            if not self.const_mask:
                assert tuple(f.shape) == self.mask.shape, "Data must have same shape as the mask!"
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        dev = b.device
        inv_fish = torch.as_tensor(self.inv_fish_ideal, device=dev)
        norm = torch.as_tensor(b.volume / float(b.gridsize.prod()) / self.sym_factor, device=dev)
        main = torch.cuda.current_stream(dev)
        side = torch.cuda.Stream(device=dev)
        rd = b.real_dtype
        bufs = [torch.empty(tuple(int(n) for n in b.gridsize), dtype=rd, device=dev) for _ in range(2)]
        ready = [torch.cuda.Event() for _ in range(2)]
        free = [torch.cuda.Event() for _ in range(2)]
        out = torch.empty((len(fields), self.N_bins), dtype=torch.float64).pin_memory()

        def upload(i):
            s = i % 2
            with torch.cuda.stream(side):
                if i >= 2:
                    side.wait_event(free[s])
                src = fields[i] if isinstance(fields[i], torch.Tensor) else torch.from_numpy(np.ascontiguousarray(fields[i]))
                bufs[s].copy_(src, non_blocking=True)
                ready[s].record(side)

        if fields:
            upload(0)
        for i in range(len(fields)):
            if i + 1 < len(fields):
                upload(i + 1)
            s = i % 2
            main.wait_event(ready[s])
            B3 = self._bk_cubic(bufs[s], 'ideal')
            free[s].record(main)
            out[i].copy_(inv_fish @ (B3 * norm), non_blocking=True)
        main.synchronize()
        return out.numpy()

    # ------------------------------------------------------------------------------
    # Monte Carlo Fisher (bspec.py:473-693), FP64
    # ------------------------------------------------------------------------------
    def _mask_device(self):
        return self.base.to_device_grid(('bk_mask', id(self)), lambda: self.mask, torch.float64)

    def _pointing(self):
        """The pointing matrix of the varying mask, with the integral constraint asked for."""
        if self._pt is None:
            kind = 'RIC' if self.add_RIC else ('GIC' if self.add_GIC else 'mask')
            self._pt = pointing.Pointing(self.base, self._mask_device(), getattr(self, 'mask_IC', None), kind,
                                         getattr(self, 'radial_bins_RIC', None))
        return self._pt

    def _modes_of_shell(self, s):
        if self._shell_modes is None:
            b = self.base
            mk = b.modk_grid.reshape(-1)
            ks = self.k_bins_squeeze
            self._shell_modes = [torch.as_tensor(np.nonzero((mk >= ks[i]) & (mk < ks[i + 1]))[0].astype(np.int64),
                                                 device=b.device) for i in range(self.Nk_squeeze)]
        return self._shell_modes[s]

    def _apply_filter_spectra(self, Q, prescaled):
        """S^-1 P on a batch of half spectra: mask_mean * Q, or rfftn(P irfftn(Q)) with P the
        mask's pointing matrix (bspec.py:499-505); in place.
        `prescaled`: Q already carries mask_mean (constant mask) or 1/N^3 (varying mask)."""
        b = self.base
        if self.const_mask:
            return Q
        qr = b.fft_c2r(Q)
        self._pointing()(qr, False, out=qr)
        b.n_FFTs_reverse += Q.shape[0]
        b.n_FFTs_forward += Q.shape[0]
        return b.fft_r2c(qr, out=Q)

    def _all_g(self, w1, w2):
        nks = self.Nk_squeeze
        if self.base.sightline == 'local' and self.lmax > 0:
            # l > 0 maps from the harmonic transform of each weighted map (bspec.py:548-577)
            return (self._g_maps_local(w1, None, 1.0, coarse=False), self._g_maps_local(w2, None, 1.0, coarse=False))
        specs = [(bb, l, 0, 1.0) for l in range(0, self.lmax + 1, 2) for bb in range(nks)]
        G1 = self._binned_maps(w1, specs, None, torch.float64, coarse=False)
        G2 = self._binned_maps(w2, specs, None, torch.float64, coarse=False)
        return G1, G2

    def _key_fts(self, G1, G2, keys):
        """FT[g1_0,A g1_l,B - g2_0,A g2_l,B] for keys (A, B, l) as a batch of half spectra."""
        b = self.base
        nks = self.Nk_squeeze
        pairs = [(A, (l // 2) * nks + B) for (A, B, l) in keys]
        prods = nat.pair_products(G1, G1, pairs, Z=G2, U=G2)
        b.n_FFTs_forward += len(keys)
        return b.fft_r2c(prods)

    def _filter_rows(self, R, xi, mask_shot):
        """S^-1 P (xi None) or its covariance form S^-1 [P xi P^dag + N] S^-dag on a block of
        half spectra prescaled as `_apply_filter_spectra` takes them (1 instead of the mask
        mean for the covariance form), 64 maps at a time; in place."""
        if self._custom_sinv:
            # the caller's S^-1, one map at a time as the reference applies it (bspec.py:499-519);
            # R holds unscaled spectra here
            b = self.base
            for r in range(R.shape[0]):
                if xi is not None:
                    x = R[r] if self.const_mask else b.to_real(R[r])
                    R[r] = covariance.cov_custom(b, x, not self.const_mask, xi, self.const_mask,
                                                 getattr(self, "mask_mean", None),
                                                 None if self.const_mask else self._pointing(), mask_shot,
                                                 lambda y, i, o: self._sinv(y, i, o),
                                                 lambda y, i, o: self._sinv(y, i, o, transpose=True))
                elif self.const_mask:
                    R[r] = self._sinv(R[r], 'fourier', 'fourier') * float(self.mask_mean)
                else:
                    R[r] = self._sinv(self._pointing()(b.to_real(R[r]), False), 'real', 'fourier')
            return R
        if xi is None:
            return self._apply_filter_spectra(R, True)
        m = None if self.const_mask else self._pointing()
        for c0 in range(0, R.shape[0], 64):
            covariance.cov_rows(self.base, R[c0:c0 + 64], xi, self.const_mask, getattr(self, "mask_mean", None), m,
                                mask_shot)
        return R

    def _fisher_from_fields(self, a1, a2, xi=None, mask_shot=None):
        """Fisher contribution of one GRF pair (bspec.py:473-676); with xi (device grids of
        a covariance spectrum) and mask_shot (device two-point shot mask, varying masks) the
        covariance contribution (bspec.py:447-471)."""
        b = self.base
        local = b.sightline == 'local' and self.lmax > 0
        ab = self.all_bins
        ks = self.k_bins_squeeze
        F64 = nat.PB_F64
        nh = b.nhalf
        invN = 1.0 / b.nreal
        # --- Q[A^-1 a] (compute_Q 'Ainv', bspec.py:536-640)
        ainv_w = b.to_device_grid('ainv', b._ainv_weight, torch.float64)
        w = torch.empty((2,) + b.nhalf_shape, dtype=torch.complex128, device=b.device)
        nat.spectral_filter(b.grid, F64, a1, w[0:1], [(0, -1.0, np.inf, 0, 0, 1.0, 1)], w=ainv_w)
        nat.spectral_filter(b.grid, F64, a2, w[1:2], [(0, -1.0, np.inf, 0, 0, 1.0, 1)], w=ainv_w)
        G1, G2 = self._all_g(w[0], w[1])
        keys = sorted({(int(r[0]), int(r[1]), 0) for r in ab} | {(int(r[1]), int(r[2]), int(r[3])) for r in ab} |
                      {(int(r[0]), int(r[2]), int(r[3])) for r in ab})
        kpos = {k: i for i, k in enumerate(keys)}
        FT = self._key_fts(G1, G2, keys)
        del G1, G2
        qs = 1.0 if self._custom_sinv else (invN if not self.const_mask else (1.0 if xi is not None else self.mask_mean))
        Q = torch.empty((self.N_bins,) + b.nhalf_shape, dtype=torch.complex128, device=b.device)
        # leg b3 carries L_l; with the local sightline that leg is applied in real space below
        leg1 = [(kpos[(r[0], r[1], 0)], ks[r[2]], ks[r[2] + 1], 0 if local else r[3], 0,
                 0.0 if (local and r[3] > 0) else qs, 0) for r in ab.tolist()]
        leg2 = [(kpos[(r[1], r[2], r[3])], ks[r[0]], ks[r[0] + 1], 0, 0, qs, 0) for r in ab.tolist()]
        leg3 = [(kpos[(r[0], r[2], r[3])], ks[r[1]], ks[r[1] + 1], 0, 0, qs, 0) for r in ab.tolist()]
        nat.spectral_filter(b.grid, F64, FT, Q, leg1, src_stride=nh)
        nat.spectral_filter(b.grid, F64, FT, Q, leg2, src_stride=nh, accumulate=True)
        nat.spectral_filter(b.grid, F64, FT, Q, leg3, src_stride=nh, accumulate=True)
        if local:
            # Q += FT[sum_m Y_lm(x) IFT(Y_lm(k) Theta_b3 FT_AB0)] for the rows of multipole l
            # (bspec.py:621-631), batched over the rows
            harm = b.harmonics
            for l in range(2, self.lmax + 1, 2):
                rows = [i for i, r in enumerate(ab.tolist()) if r[3] == l]
                if not rows:
                    continue
                bands = [(kpos[(int(ab[i, 0]), int(ab[i, 1]), 0)], ks[ab[i, 2]], ks[ab[i, 2] + 1], 0, 0, invN, 1)
                         for i in rows]
                yr = harm._grid('r', l, torch.float64)
                yk = harm._grid('k', l, torch.float64)
                acc = torch.zeros((len(rows),) + tuple(int(n) for n in b.gridsize), dtype=torch.float64,
                                  device=b.device)
                T = torch.empty((len(rows),) + b.nhalf_shape, dtype=torch.complex128, device=b.device)
                for mi in range(yr.shape[0]):
                    nat.spectral_filter(b.grid, F64, FT, T, bands, src_stride=nh, w=yk[mi])
                    acc.addcmul_(b.fft_c2r(T), yr[mi])
                    b.n_FFTs_reverse += len(rows)
                b.n_FFTs_forward += len(rows)
                idx = torch.as_tensor(rows, device=b.device)
                Q[idx] = Q[idx] + b.fft_r2c(acc) * qs
        del FT
        Q = self._filter_rows(Q, xi, mask_shot)
        # --- rows from Q[S^-1 P a] (compute_Q 'Sinv', bspec.py:528-597)
        if self._custom_sinv:
            ws = torch.stack([a1.reshape(b.nhalf_shape), a2.reshape(b.nhalf_shape)]).to(torch.complex128)
            ws = self._filter_rows(ws, xi, mask_shot)
        elif self.const_mask:
            ws = torch.empty((2,) + b.nhalf_shape, dtype=torch.complex128, device=b.device)
            nat.spectral_filter(b.grid, F64, a1, ws[0:1], [(0, -1.0, np.inf, 0, 0, qs, 0)])
            nat.spectral_filter(b.grid, F64, a2, ws[1:2], [(0, -1.0, np.inf, 0, 0, qs, 0)])
            if xi is not None:
                ws = self._filter_rows(ws, xi, mask_shot)
        else:
            ws = torch.empty((2,) + b.nhalf_shape, dtype=torch.complex128, device=b.device)
            nat.spectral_filter(b.grid, F64, a1, ws[0:1], [(0, -1.0, np.inf, 0, 0, invN, 0)])
            nat.spectral_filter(b.grid, F64, a2, ws[1:2], [(0, -1.0, np.inf, 0, 0, invN, 0)])
            b.n_FFTs_reverse += 2
            ws = self._filter_rows(ws, xi, mask_shot)
        G1, G2 = self._all_g(ws[0], ws[1])
        skeys = sorted({(int(r[0]), int(r[2]), int(r[3])) for r in ab})
        spos = {k: i for i, k in enumerate(skeys)}
        FTs = self._key_fts(G1, G2, skeys)
        del G1, G2
        fish = torch.zeros((self.N_bins, self.N_bins), dtype=torch.float64, device=b.device)
        scale = 0.5 * b.volume / float(b.gridsize.prod()) ** 2
        for s in range(self.Nk_squeeze):
            rows = np.nonzero(ab[:, 1] == s)[0]
            if len(rows) == 0:
                continue
            modes = self._modes_of_shell(s)
            for r0 in range(0, len(rows), 32):
                rr = rows[r0:r0 + 32]
                rk = [spos[(int(ab[i, 0]), int(ab[i, 2]), int(ab[i, 3]))] for i in rr]
                nat.shell_rows(b.grid, FTs, Q, modes, rk, rr, scale, fish, b.ws)
        sym = self.base.to_device_grid(('bk_sym2', id(self)), lambda: np.outer(self.sym_factor, self.sym_factor),
                                       torch.float64)
        return fish / sym

    def compute_fisher_contribution(self, seed, verb=False):
        """Fisher contribution of one GRF pair with the reference's noise draws (bspec.py:441-445)."""
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        b = self.base
        r1 = b.reference_noise(seed + int(1e7))
        r2 = b.reference_noise(seed + int(2e7))
        a1 = b.grf_from_noise(torch.as_tensor(r1[0], device=b.device), torch.as_tensor(r1[1], device=b.device))
        a2 = b.grf_from_noise(torch.as_tensor(r2[0], device=b.device), torch.as_tensor(r2[1], device=b.device))
        return self._fisher_from_fields(a1, a2).cpu().numpy()

    def compute_fisher(self, N_it, verb=False, *, group=None, noise='reference'):
        """Mean Fisher over seeds 0..N_it-1 (bspec.py:678-693).  Under an initialised
        torch.distributed process group (`group`, default the world) the seeds are shared
        round-robin over the ranks; every rank returns the same matrix, summed in seed
        order exactly as the one-process loop sums it.
        noise='reference': the reference's own MT19937 draws per seed (identical inputs);
        noise='philox': white noise drawn on the device (Philox, keyed by seed + 1e7 and
        seed + 2e7) and each realisation replayed from one captured CUDA graph."""
        assert noise in ('reference', 'philox'), "noise must be 'reference' or 'philox'"
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        b = self.base
        feed = None
        if noise == 'reference' and realisations.prefetch_pays(2 * N_it, b.gridsize):
            # the reference's two draws per seed for this rank's seeds, made ahead on host workers
            rank, size = realisations.world(group)
            feed = realisations.noise_pool(b.gridsize).stream(
                [s + off for s in realisations.seeds_of_rank(N_it, rank, size) for off in (int(1e7), int(2e7))])

        def contrib(seeds):
            if noise == 'philox' and self._custom_sinv:
                # a caller's S^-1 may synchronise or allocate on the host: no graph capture
                return torch.cat([self._fisher_from_fields(b.grf_philox(np.asarray([s], dtype=np.int64) + int(1e7)),
                                                           b.grf_philox(np.asarray([s], dtype=np.int64) + int(2e7)))[None]
                                  for s in seeds])
            if noise == 'philox':
                if self._captured is None:
                    self._captured = realisations.CapturedBatch(
                        lambda sd: self._fisher_from_fields(b.grf_philox(sd + int(1e7)),
                                                            b.grf_philox(sd + int(2e7)))[None], 1, b)
                return torch.cat([self._captured.run([s]) for s in seeds])
            if feed is not None:
                out = []
                for _ in seeds:
                    nre, nim = feed.take(2, b.device)
                    out.append(self._fisher_from_fields(b.grf_from_noise(nre[0], nim[0]),
                                                        b.grf_from_noise(nre[1], nim[1]))[None])
                return torch.cat(out)
            return np.stack([self.compute_fisher_contribution(s, verb=verb) for s in seeds])

        def progress(seeds):
            for s in seeds:
                if s % 5 == 0:
                    print("Computing Fisher contribution %d of %d" % (s + 1, N_it))

        fish = realisations.mc_mean(contrib, N_it, (self.N_bins, self.N_bins), self.base.device, group=group,
                                    progress=progress).cpu().numpy()
        self.fish = fish
        self.inv_fish = np.linalg.inv(fish)
        return fish

    def Bk_unwindowed(self, data, fish=[], include_linear_term=True, verb=False):
        """Unwindowed estimator (bspec.py:863-893)."""
        if len(fish) != 0:
            self.fish = fish
            self.inv_fish = np.linalg.inv(fish)
        if not hasattr(self, 'inv_fish'):
            raise Exception("Need to compute Fisher matrix first!")
        Bk_num = self.Bk_numerator(data, include_linear_term=include_linear_term, verb=verb)
        Bk_out = np.matmul(self.inv_fish, Bk_num)
        Bk_dict = {}
        index = 0
        for l in range(0, self.lmax + 1, 2):
            Bk_dict['b%s' % l] = Bk_out[index:index + self.N3]
            index += self.N3
        return Bk_dict

    def compute_shot_contribution(self, seed, verb=False, data=None, data2=None, cubic_only=False):
        """Shot-noise contribution of one pair of GRFs of spectrum 1/P_fid (bspec.py:695-861;
        with the local sightline every map set's l > 0 maps come from the harmonic transform): the cubic term from the maps of S^-1 a1, S^-1 a2 and the
        shot-masked product (A^-1 a1)(A^-1 a2), and unless cubic_only the quadratic term from
        the data's maps with those of (A^-1 a_i) d2.  Returns quadratic - 2 cubic."""
        if not cubic_only:
            assert data is not None, "Must supply data to compute the quadratic shot-noise contribution!"
            if data2 is None:
                print("## Caution: assuming uniform weights!")
                data2 = data
            if not self.const_mask:
                assert data.shape == self.mask.shape, "Data must have same shape as the mask!"
            for dd in (data, data2):
                if not isinstance(dd, torch.Tensor):
                    assert type(dd[0, 0, 0]) in [np.float32, np.float64], "Data must be of type float32 or float64!"
        else:
            print("## Caution: Dropping quadratic (~ P(k)/n) term!")
        assert hasattr(self, 'mask_shot'), "Must supply triply-weighted mask to compute the shot-noise contribution!"
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        b = self.base
        dev = b.device
        rd = b.real_dtype
        F64 = nat.PB_F64
        PkA = [b.Pfid[0], 1. / b.Pfid[1]]
        a = []
        for off in (int(1e7), int(2e7)):
            re, im = b.reference_noise(seed + off)
            a.append(b.grf_from_noise(torch.as_tensor(re, device=dev), torch.as_tensor(im, device=dev), Pk_input=PkA))
        # A^-1 a_i with the base fiducial spectrum in place of 1/P (bspec.py:772, 779-780)
        r = [b.applyAinv(ai, invPk0_grid=b.Pk0_grid, input_type='fourier', output_type='real') for ai in a]
        mshot = b.to_device_grid(('bk_mask_shot', id(self)), lambda: self.mask_shot, torch.float64)
        n = self.Nl * self.Nk_squeeze
        X = torch.empty((3 * n,) + tuple(self.map_grid), dtype=rd, device=dev)
        cd = torch.complex128 if rd == torch.float64 else torch.complex64
        sets = [X[i * n:(i + 1) * n] for i in range(3)]
        perms = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))

        def maps_of(spec, out, w=None):
            self._g_maps(spec if spec.dtype == cd else spec.to(cd), w, 1.0, out=out)

        def product_spectrum(x, y, z=None):
            prod = nat.elementwise(nat.PB_EW_MUL, x, y)
            if z is not None:
                nat.elementwise(nat.PB_EW_MUL, prod, z, out=prod, y_period=b.nreal)
            if self._custom_sinv:                                        # bspec.py:781-785
                return self._sinv(prod, 'real', 'fourier')
            return b.to_fourier(prod)

        if self._custom_sinv:                                            # bspec.py:788-790
            a = [self._sinv(ai, 'fourier', 'fourier') for ai in a]
        maps_of(a[0], sets[0])
        maps_of(a[1], sets[1])
        maps_of(product_spectrum(r[0], r[1], mshot), sets[2])
        norm = b.volume / float(b.gridsize.prod()) / self.sym_factor
        cubic = self._set_sums('bshot', X, n, perms).cpu().numpy() * norm / 6.
        if cubic_only:
            return cubic
        w = None
        if self._custom_sinv:                                            # bspec.py:733-742
            xk = self._sinv_data(data)
        else:
            xk = b.to_fourier(b.as_device(data))
            if b.pixel_window != 'none':
                w = b.to_device_grid(('bk_invwin', id(self)), lambda: self._inv_window(), xk.real.dtype)
        d2 = b.as_device(data2, torch.float64)
        # (g, a1-maps, D) in the three sets, then (a2-maps, g, E)
        maps_of(xk, sets[1], w)
        maps_of(product_spectrum(r[0], d2), sets[2])
        quad = self._set_sums('bshot', X, n, perms)
        maps_of(a[1], sets[0])
        maps_of(product_spectrum(r[1], d2), sets[2])
        quad = quad + self._set_sums('bshot', X, n, perms)
        quad = 0.5 * quad.cpu().numpy() * norm / 2.
        return quad - 2. * cubic

    def compute_covariance_contribution(self, seed, Pk_cov, verb=False, mask_shot_2pt=None):
        """Contribution of one GRF pair to the Gaussian covariance of the unwindowed
        bispectrum (bspec.py:447-471): the Fisher computation with S^-1 P replaced by
        S^-1 [P xi P^dag + N] S^-dag, xi the correlation of Pk_cov = [k, P0(, P2(, P4))]
        (no shot noise) and N the two-point shot mask (mask_shot_2pt, else the bispectrum's
        mask_shot; the mask mean for a constant mask).  Same noise as
        compute_fisher_contribution."""
        if (not self.const_mask) and (mask_shot_2pt is None):
            assert getattr(self, 'mask_shot', None) is not None, \
                "Must supply a shot-noise mask to compute the shot-noise contribution!"
            print("## Caution: assuming the same shot-noise mask for the power spectrum and bispectrum!")
            self.mask_shot_2pt = self.mask_shot
        elif mask_shot_2pt is not None:
            self.mask_shot_2pt = np.asarray(mask_shot_2pt).astype(np.float64)
        else:
            self.mask_shot_2pt = None
        assert len(Pk_cov) != 0, "Must provide fiducial power spectrum if computing covariance!"
        assert len(np.asarray(Pk_cov).shape) == 2, "Pk should contain k and P_0 (and optionally P_2, P_4) columns"
        assert len(Pk_cov) in [2, 3, 4], "Pk should contain k and P_0 (and optionally P_2, P_4) columns"
        if not hasattr(self, 'sym_factor'):
            self._compute_symmetry_factor()
        b = self.base
        ms = None
        if not self.const_mask:
            ms = torch.as_tensor(np.ascontiguousarray(self.mask_shot_2pt), dtype=torch.float64, device=b.device)
        xi = covariance.xi_grids(b, Pk_cov)
        r1 = b.reference_noise(seed + int(1e7))
        r2 = b.reference_noise(seed + int(2e7))
        a1 = b.grf_from_noise(torch.as_tensor(r1[0], device=b.device), torch.as_tensor(r1[1], device=b.device))
        a2 = b.grf_from_noise(torch.as_tensor(r2[0], device=b.device), torch.as_tensor(r2[1], device=b.device))
        return self._fisher_from_fields(a1, a2, xi=xi, mask_shot=ms).cpu().numpy()


_TC_OK = None


def tc_available():
    """True when the tensor-core contraction is built for this device (sm_100)."""
    global _TC_OK
    if _TC_OK is None:
        try:
            cap = torch.cuda.get_device_capability()
            _TC_OK = cap[0] == 10 and nat.tc_built()
        except Exception:
            _TC_OK = False
    return _TC_OK
