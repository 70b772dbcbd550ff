"""PolyBin3D base class, backend='cuda' (mirrors PolyBin3D/base.py).

Geometry (k-grids, windows, fiducial spectrum) follows base.py:20-144; the grids are
numpy arrays built on first access, and their device copies are made once.  Transforms
run through cuFFT plans of the C ABI (pb_fft_*), r2c forward unnormalised and c2r with
numpy's 1/N^3 (base.py:176-229), counted in n_FFTs_forward / n_FFTs_reverse.
"""
import os

import numpy as np
import scipy.interpolate
import torch

from . import _native as nat

PRECISIONS = ("fp64", "mixed")


class PolyBin3D:
    """Base class for the CUDA backend of PolyBin3D.

    Inputs as in the reference (base.py:7-19).  `backend` must be 'cuda'.  Keyword-only
    additions:
    - precision: 'fp64' (FP64 FFTs and sums; default, bit-for-bit binning and ~1e-12
      agreement with the reference) or 'mixed' (FP32 transforms and maps, FP64 sums).
      Monte Carlo Fisher matrices, ideal Fisher matrices and symmetry factors always run
      in FP64.
    - device: CUDA device (default: the current one).
    """

    def __init__(self, boxsize, gridsize, Pk=None, boxcenter=None, pixel_window='none', backend='cuda',
                 nthreads=None, sightline='global', real_fft=True, *, precision='fp64', device=None, verb=True):
        self.backend = backend
        self.nthreads = nthreads if nthreads is not None else os.cpu_count()
        self.sightline = sightline
        self.pixel_window = pixel_window
        self.real_fft = real_fft
        if backend != 'cuda':
            raise Exception("polybin3d_b200 implements backend='cuda' only; use the reference package "
                            "for 'fftw', 'mkl' and 'jax'")
        if precision not in PRECISIONS:
            raise ValueError("precision must be one of %s" % (PRECISIONS,))
        self.precision = precision

        # box size, centre and grid (base.py:31-54)
        if type(boxsize) == float:
            self.boxsize = np.asarray([boxsize, boxsize, boxsize])
        else:
            assert len(boxsize) == 3, "Need to specify x, y, z boxsize"
            self.boxsize = np.asarray(boxsize, dtype=np.float64)
        if boxcenter is None:
            self.boxcenter = np.zeros(3)
        elif type(boxcenter) == float:
            self.boxcenter = np.asarray([boxcenter, boxcenter, boxcenter])
        else:
            assert len(boxcenter) == 3, "Need to specify x, y, z boxcenter"
            self.boxcenter = np.asarray(boxcenter)
        if type(gridsize) == int:
            self.gridsize = np.asarray([gridsize, gridsize, gridsize], dtype=int)
        else:
            assert len(gridsize) == 3, "Need to specify n_x, n_y, n_z gridsize"
            self.gridsize = np.asarray(gridsize, dtype=int)
        if real_fft and gridsize[2] % 2 != 0:
            raise Exception("Last dimension of grid must be even for real-to-complex FFTs.")
        if not real_fft:
            raise NotImplementedError("backend='cuda' implements real-to-complex transforms (real_fft=True) only")

        assert self.sightline in ['local', 'global'], "Sight-line must be 'local' or 'global'"
        if self.sightline == 'global':
            assert np.abs(self.boxcenter).sum() == 0., "Global sightlines should only be used for simulation data!"
        if self.sightline == 'local':
            assert np.abs(self.boxcenter).sum() != 0., "Local sightlines should only be used for lightcone data!"
        # line of sight of the mu grid: the z axis, or the direction of the box centre
        # (base.py:111-114); the local-sightline multipoles also use the real harmonics of
        # the voxel positions (harmonics.py)
        if self.sightline == 'global':
            self.sight_vector = np.asarray([0., 0., 1.])
        else:
            self.sight_vector = self.boxcenter / np.sqrt(np.sum(self.boxcenter ** 2))

        # derived parameters (base.py:63-74)
        self.volume = self.boxsize.prod()
        self.kF = 2. * np.pi / self.boxsize
        self.kNy = self.gridsize * self.kF * 0.5
        if (np.asarray(Pk) == None).all():  # noqa: E711  (reference test, base.py:68)
            k_tmp = np.arange(0., np.max(self.kNy) * 2, np.min(self.kF) / 10.)
            self.Pfid = np.asarray([k_tmp, 1. + 0. * k_tmp])
            self._unit_pk = True
        else:
            assert len(Pk) == 2, "Pk should contain k and P_0(k) columns"
            self.Pfid = np.asarray(Pk)
            self._unit_pk = False
        self.kmin, self.kmax = np.min(self.Pfid[0, 0]), np.max(self.Pfid[0, -1])

        self.pixel_windows = ['none', 'cic', 'tsc', 'pcs', 'interlaced-cic', 'interlaced-tsc', 'interlaced-pcs']
        assert self.pixel_window in self.pixel_windows, "Unknown pixel window '%s' supplied!" % pixel_window
        if verb:
            print("\n# Dimensions: [%.2e, %.2e, %.2e] Mpc/h" % tuple(self.boxsize))
            print("# Center: [%.2e, %.2e, %.2e] Mpc/h" % tuple(self.boxcenter))
            print("# Line-of-sight: %s" % self.sightline)
            print("# Cartesian grid: [%d, %d, %d]" % tuple(self.gridsize))
            print("# Fundamental frequency: [%.4f, %.4f, %.4f] h/Mpc" % tuple(self.kF))
            print("# Nyquist frequency: [%.3f, %.3f, %.3f] h/Mpc" % tuple(self.kNy))
            print("# Pixel window: %s" % self.pixel_window)
            print("# Using CUDA backend (%s)" % precision)

        # device set-up
        nat.require_cuda()
        self.device = torch.device(device) if device is not None else torch.device('cuda', torch.cuda.current_device())
        self.grid = self.grid_of(self.gridsize)
        self.nhalf_shape = (int(self.gridsize[0]), int(self.gridsize[1]), int(self.gridsize[2]) // 2 + 1)
        self.nreal = int(self.gridsize.prod())
        self.nhalf = int(np.prod(self.nhalf_shape))
        self.ws = nat.Workspace(self.device)
        self._plans = {}
        self._dev = {}
        self._host = {}
        self.n_FFTs_forward = 0
        self.n_FFTs_reverse = 0

    # ------------------------------------------------------------------------------
    # host geometry, built on first use (base.py:76-131)
    # ------------------------------------------------------------------------------
    def _k_arrs(self):
        k_arrs = [np.fft.fftshift(np.arange(-self.gridsize[i] // 2, self.gridsize[i] // 2)) * self.kF[i]
                  for i in range(2)]
        k_arrs += [np.arange(0, self.gridsize[2] // 2 + 1) * self.kF[2]]
        return k_arrs

    def _lazy(self, name, fn):
        if name not in self._host:
            self._host[name] = fn()
        return self._host[name]

    @property
    def k_grids(self):
        return self._lazy('k_grids', lambda: np.meshgrid(*self._k_arrs(), indexing='ij'))

    @property
    def modk_grid(self):
        kg = self.k_grids
        return self._lazy('modk', lambda: np.sqrt(kg[0] ** 2 + kg[1] ** 2 + kg[2] ** 2))

    @property
    def degeneracy_factor(self):
        return self._lazy('deg', lambda: np.asarray(1. + (self.k_grids[2] > 0), dtype=np.float64))

    @property
    def muk_grid(self):
        def f():
            mk = self.modk_grid
            mu = np.zeros(mk.shape)
            nz = mk != 0
            mu[nz] = np.sum(self.sight_vector[:, None] * np.asarray(self.k_grids)[:, nz], axis=0) / mk[nz]
            return mu
        return self._lazy('muk', f)

    @property
    def r_grids(self):
        """Voxel positions relative to the observer: fftshift order plus the box centre
        (base.py:75-79); local sightline only."""
        assert self.sightline == 'local', "r_grids are defined for the local sightline"

        def f():
            r_arrs = [np.fft.fftshift(np.arange(-self.gridsize[i] // 2, self.gridsize[i] // 2)) * self.boxsize[i]
                      / self.gridsize[i] + self.boxcenter[i] for i in range(3)]
            return np.meshgrid(*r_arrs, indexing='ij')
        return self._lazy('rgrids', f)

    @property
    def harmonics(self):
        """Device real-harmonic grids of this box (local-sightline multipoles)."""
        if getattr(self, '_harm', None) is None:
            from .harmonics import Harmonics
            self._harm = Harmonics(self)
        return self._harm

    def _pixel_window_1d(self, k):
        """Pixel window functions including first-order alias corrections (base.py:231-254)."""
        if self.pixel_window == 'cic':
            s = np.sin(k) ** 2.
            v = (1. - 2. / 3. * s) ** 0.5
        elif self.pixel_window == 'tsc':
            s = np.sin(k) ** 2.
            v = (1. - s + 2. / 15 * s ** 2.) ** 0.5
        elif self.pixel_window == 'pcs':
            s = np.sin(k) ** 2.
            v = (1. - 4. / 3. * s + 2. / 5. * s ** 2 - 4. / 315. * s ** 3) ** 0.5
        elif self.pixel_window == 'interlaced-cic':
            s = np.sinc(k / np.pi)
            v = np.ones_like(s)
            v[s != 0.] = s[s != 0.] ** 2.
        elif self.pixel_window == 'interlaced-tsc':
            v = np.sinc(k / np.pi) ** 3.
        elif self.pixel_window == 'interlaced-pcs':
            v = np.sinc(k / np.pi) ** 4.
        else:
            raise Exception("Unknown window function '%s' supplied!" % self.pixel_window)
        return v

    @property
    def pixel_window_grid(self):
        if self.pixel_window == 'none':
            raise AttributeError("pixel_window_grid is only defined for a pixel window")

        def f():
            ka = self._k_arrs()
            w1 = [self._pixel_window_1d(np.pi / self.gridsize[i] * ka[i] / self.kF[i]) for i in range(3)]
            return np.asarray(np.meshgrid(*w1, indexing='ij')).prod(axis=0)
        return self._lazy('window', f)

    def _pk_grids(self):
        Pk0 = scipy.interpolate.interp1d(self.Pfid[0], self.Pfid[1], bounds_error=False,
                                         fill_value=0.)(self.modk_grid)
        invPk0 = np.zeros(self.modk_grid.shape, dtype=np.float64)
        good = (Pk0 != 0) & np.isfinite(Pk0)
        invPk0[good] = 1. / Pk0[good]
        Pk0[~np.isfinite(Pk0)] = 0.
        invPk0[self.modk_grid == 0] = 1.
        Pk0[self.modk_grid == 0] = 1.
        return Pk0, invPk0

    @property
    def Pk0_grid(self):
        return self._lazy('pk', self._pk_grids)[0]

    @property
    def invPk0_grid(self):
        return self._lazy('pk', self._pk_grids)[1]

    # ------------------------------------------------------------------------------
    # device buffers
    # ------------------------------------------------------------------------------
    @property
    def real_dtype(self):
        return torch.float64 if self.precision == 'fp64' else torch.float32

    @property
    def complex_dtype(self):
        return torch.complex128 if self.precision == 'fp64' else torch.complex64

    def to_device_grid(self, name, fn, dtype):
        """Upload a host per-mode (or per-voxel) grid once and cache it by (name, dtype)."""
        key = (name, dtype)
        if key not in self._dev:
            arr = fn()
            self._dev[key] = None if arr is None else torch.as_tensor(np.ascontiguousarray(arr), dtype=dtype,
                                                                      device=self.device)
        return self._dev[key]

    def real_zeros(self, size=None, numpy=False, dtype=None):
        shape = [] if size is None else ([size] if type(size) == int else list(size))
        shape += [int(g) for g in self.gridsize]
        if numpy:
            return np.zeros(shape, dtype=np.float64)
        return torch.zeros(shape, dtype=dtype or self.real_dtype, device=self.device)

    def complex_zeros(self, size=None, numpy=False, dtype=None):
        shape = [] if size is None else ([size] if type(size) == int else list(size))
        shape += list(self.nhalf_shape)
        if numpy:
            return np.zeros(shape, dtype=np.complex128)
        return torch.zeros(shape, dtype=dtype or self.complex_dtype, device=self.device)

    def as_device(self, data, dtype=None):
        """numpy or torch -> contiguous device tensor of `dtype` (real maps)."""
        dtype = dtype or self.real_dtype
        if isinstance(data, torch.Tensor):
            return data.to(device=self.device, dtype=dtype).contiguous()
        return torch.as_tensor(np.ascontiguousarray(data), device=self.device).to(dtype).contiguous()

    # ------------------------------------------------------------------------------
    # transforms (base.py:176-229)
    # ------------------------------------------------------------------------------
    def grid_of(self, dims):
        """C-ABI grid descriptor with this box's fundamental frequencies and real dims `dims`."""
        g = nat.PBGrid()
        for i in range(3):
            g.n[i] = int(dims[i])
            g.kf[i] = float(self.kF[i])
        g.flags = 0
        if self.sightline == 'local':
            # mu = (k . n)/|k| with n the unit vector to the box centre (base.py:111-116)
            g.flags = nat.PB_GRID_LOS
            for i in range(3):
                g.los[i] = float(self.sight_vector[i])
        return g

    def _plan(self, batch, precision, direction, dims=None):
        dims = tuple(int(d) for d in (self.gridsize if dims is None else dims))
        key = (dims, batch, precision, direction)
        p = self._plans.get(key)
        if p is None:
            p = nat.FFTPlan(self.grid_of(dims), batch, precision, direction)
            self._plans[key] = p
        return p

    def fft_r2c(self, x, out=None):
        """Unnormalised r2c of real maps x (..., n0, n1, n2) -> half spectra (raw call, no count)."""
        prec = nat.precision_of(x.dtype)
        dims = tuple(x.shape[-3:])
        batch = int(np.prod(x.shape[:-3])) if x.dim() > 3 else 1
        cd = torch.complex128 if prec == nat.PB_F64 else torch.complex64
        hs = (dims[0], dims[1], dims[2] // 2 + 1)
        out = torch.empty(tuple(x.shape[:-3]) + hs, dtype=cd, device=self.device) if out is None else out
        p = self._plan(batch, prec, nat.PB_FFT_R2C, dims)
        p.exec(x, out, self.ws.get(p.ws_bytes, "fft"))
        return out

    def fft_c2r(self, k, out=None):
        """Unnormalised c2r of half spectra (destroys k) -> real maps (raw call, no count).
        The real grid is (n0, n1, 2*(n2h-1)) from the spectrum's shape."""
        prec = nat.precision_of(k.dtype)
        hs = tuple(k.shape[-3:])
        dims = (hs[0], hs[1], 2 * (hs[2] - 1))
        batch = int(np.prod(k.shape[:-3])) if k.dim() > 3 else 1
        rd = torch.float64 if prec == nat.PB_F64 else torch.float32
        out = torch.empty(tuple(k.shape[:-3]) + dims, dtype=rd, device=self.device) if out is None else out
        p = self._plan(batch, prec, nat.PB_FFT_C2R, dims)
        p.exec(k, out, self.ws.get(p.ws_bytes, "fft"))
        return out

    def to_fourier(self, _input_rmap):
        """Transform from real- to Fourier-space (numpy rfftn convention)."""
        x = self.as_device(_input_rmap) if not isinstance(_input_rmap, torch.Tensor) else _input_rmap.contiguous()
        self.n_FFTs_forward += int(np.prod(x.shape[:-3])) if x.dim() > 3 else 1
        return self.fft_r2c(x)

    def to_real(self, _input_kmap):
        """Transform from Fourier- to real-space (numpy irfftn convention, 1/N^3)."""
        k = _input_kmap.clone()
        n = k.shape[:-3]
        self.n_FFTs_reverse += int(np.prod(n)) if len(n) else 1
        prec = nat.precision_of(k.dtype)
        nm = int(np.prod(n)) if len(n) else 1
        maps = [(i, -1.0, np.inf, 0, 0, 1.0 / self.nreal, 0) for i in range(nm)]
        kk = k.reshape((nm,) + self.nhalf_shape)
        nat.spectral_filter(self.grid, prec, kk, kk, maps, src_stride=self.nhalf)
        return self.fft_c2r(k)

    # ------------------------------------------------------------------------------
    # fields and filters (base.py:305-389)
    # ------------------------------------------------------------------------------
    def _grf_amp(self, Pk_input=None, include_pixel_window=True):
        """sqrt(P(k)) [* W(k)] on the half grid, FP64 host array."""
        if Pk_input is None or len(Pk_input) == 0:
            Pk_grid = self.Pk0_grid
        else:
            assert len(np.asarray(Pk_input).shape) == 2, "Pk should contain k and P_0, (and optionally P_2, P_4) columns"
            assert len(Pk_input) in [2, 3, 4], "Pk should contain k and P_0, (and optionally P_2, P_4) columns"
            itp = lambda y: scipy.interpolate.interp1d(Pk_input[0], y, bounds_error=False, fill_value=0.)(self.modk_grid)
            Pk_grid = itp(Pk_input[1])
            if len(Pk_input) > 2:
                Pk_grid = Pk_grid + 0.5 * (3 * self.muk_grid ** 2 - 1) * itp(Pk_input[2])
            if len(Pk_input) > 3:
                mu2 = self.muk_grid ** 2
                Pk_grid = Pk_grid + (35 * mu2 ** 2 - 30 * mu2 + 3) / 8. * itp(Pk_input[3])
        amp = np.sqrt(Pk_grid)
        if self.pixel_window != 'none' and include_pixel_window:
            amp = amp * self.pixel_window_grid
        return amp

    def grf_from_noise(self, noise_re, noise_im, Pk_input=None, include_pixel_window=True, dtype=torch.float64):
        """Half-spectrum GRF(s) from white noise (..., n0, n1, n2) FP64 device tensors."""
        key = ('amp', include_pixel_window) if not Pk_input else None
        if key is not None:
            amp = self.to_device_grid(key, lambda: self._grf_amp(None, include_pixel_window), torch.float64)
        else:
            amp = torch.as_tensor(self._grf_amp(Pk_input, include_pixel_window), device=self.device)
        nb = noise_re.shape[0] if noise_re.dim() == 4 else 1
        cd = torch.complex128 if dtype == torch.float64 else torch.complex64
        out = torch.empty(((nb,) if noise_re.dim() == 4 else ()) + self.nhalf_shape, dtype=cd, device=self.device)
        nat.grf_from_noise(self.grid, nat.precision_of(dtype), noise_re, noise_im, amp,
                           float(self.gridsize.prod() / np.sqrt(self.volume)), out)
        return out

    def grf_philox(self, seeds, out=None, include_pixel_window=True, dtype=torch.float64):
        """Half-spectrum GRFs (n_seeds, half) from white noise drawn on the device
        (Philox4x32-10 keyed by each seed): the distribution of generate_data (base.py:305-353),
        not the reference's MT19937 stream.  `seeds`: host ints or a device int64 tensor
        (a captured graph replays with whatever that tensor holds)."""
        if not isinstance(seeds, torch.Tensor):
            seeds = torch.as_tensor(np.asarray(seeds, dtype=np.int64), device=self.device)
        amp = self.to_device_grid(('amp', include_pixel_window), lambda: self._grf_amp(None, include_pixel_window),
                                  torch.float64)
        cd = torch.complex128 if dtype == torch.float64 else torch.complex64
        if out is None:
            out = torch.empty((seeds.numel(),) + self.nhalf_shape, dtype=cd, device=self.device)
        nat.grf_philox(self.grid, nat.precision_of(dtype), seeds, amp, float(self.gridsize.prod() / np.sqrt(self.volume)),
                       out)
        return out

    def reference_noise(self, seed):
        """White noise exactly as the reference draws it: np.random.seed(seed), then
        randn(*gridsize) for the real and the imaginary parts (base.py:315-316, 332)."""
        if seed is not None:
            np.random.seed(seed)
        re = np.random.randn(*self.gridsize)
        im = np.random.randn(*self.gridsize)
        return re, im

    def generate_data(self, seed=None, Pk_input=[], output_type='real', include_pixel_window=True):
        """Gaussian periodic map with the fiducial (or given) power spectrum (base.py:305-353).
        The white noise is the reference's own MT19937 draw, so outputs match it."""
        assert output_type in ['fourier', 'real'], "Valid output types are 'fourier' and 'real' only!"
        re, im = self.reference_noise(seed)
        nre = torch.as_tensor(re, device=self.device)
        nim = torch.as_tensor(im, device=self.device)
        a = self.grf_from_noise(nre, nim, Pk_input if len(Pk_input) else None, include_pixel_window)
        if output_type == 'fourier':
            return a
        return self.to_real(a)

    def applySinv_trivial(self, input_data, input_type='real', output_type='real'):
        """Trivial filter with real/Fourier conversion (base.py:355-362)."""
        if input_type == output_type:
            return input_data
        if input_type == 'fourier':
            return self.to_real(input_data)
        return self.to_fourier(input_data)

    # ------------------------------------------------------------------------------
    # harmonic transforms and the covariance kernel (base.py:391-437)
    # ------------------------------------------------------------------------------
    def _spectrum_in(self, k):
        if isinstance(k, torch.Tensor):
            return k.to(self.device)
        return torch.as_tensor(np.ascontiguousarray(k), device=self.device)

    def apply_real_harmonics(self, a_map_fourier, Ylm_real, Ylm_fourier):
        """sum_m Y_lm(r) IFT[Y_lm(k) a(k)] (base.py:391-400) as a device real map; Ylm_real
        (n_m, n0, n1, n2) and Ylm_fourier (n_m, half grid) as PSpec.Ylm_real[l] and
        PSpec.Ylm_fourier[l] hold them (numpy or device)."""
        a = self._spectrum_in(a_map_fourier)
        rd = a.real.dtype
        out = torch.zeros(tuple(int(n) for n in self.gridsize), dtype=rd, device=self.device)
        for m in range(len(Ylm_real)):
            out.addcmul_(self.to_real(a * self.as_device(Ylm_fourier[m], rd)), self.as_device(Ylm_real[m], rd))
        return out

    def apply_fourier_harmonics(self, a_map_real, Ylm_real, Ylm_fourier):
        """sum_m Y_lm(k) FT[Y_lm(r) a(r)] (base.py:402-411) as a device half spectrum."""
        x = self.as_device(a_map_real, a_map_real.dtype if isinstance(a_map_real, torch.Tensor) else torch.float64)
        cd = torch.complex128 if x.dtype == torch.float64 else torch.complex64
        out = torch.zeros(self.nhalf_shape, dtype=cd, device=self.device)
        for m in range(len(Ylm_real)):
            out.add_(self.to_fourier(x * self.as_device(Ylm_real[m], x.dtype)) * self.as_device(Ylm_fourier[m], x.dtype))
        return out

    def apply_xi(self, input_map_fourier, input_map_real=None, Ylm_real=None, Ylm_fourier=None, Pk_grid=[],
                 output_type='real'):
        """Apply xi(x, y), the correlation of the gridded spectrum Pk_grid = {l: P_l(k)}, to a
        map (base.py:413-437): P_0 X, plus for the local sightline and each further l one half
        of P_l sum_m Y_lm(k) FT[Y_lm(r) x] and one half of sum_m Y_lm(r) IFT[Y_lm(k) P_l X]."""
        X = self._spectrum_in(input_map_fourier)
        rd = X.real.dtype
        PF = X * self.as_device(Pk_grid[0], rd)
        if self.sightline == 'global' or len(Pk_grid.keys()) == 1:
            return PF if output_type == 'fourier' else self.to_real(PF)
        PR = torch.zeros(tuple(int(n) for n in self.gridsize), dtype=rd, device=self.device)
        for ell in list(Pk_grid.keys())[1:]:
            Pl = self.as_device(Pk_grid[ell], rd)
            PF = PF + 0.5 * self.apply_fourier_harmonics(input_map_real, Ylm_real[ell], Ylm_fourier[ell]) * Pl
            PR = PR + 0.5 * self.apply_real_harmonics(X * Pl, Ylm_real[ell], Ylm_fourier[ell])
        return PF + self.to_fourier(PR) if output_type == 'fourier' else self.to_real(PF) + PR

    def _ainv_weight(self):
        """invP / W^2 (0 where W = 0) on the half grid, FP64 host array."""
        w = self.invPk0_grid.copy()
        if self.pixel_window != 'none':
            W = self.pixel_window_grid
            nz = W != 0
            w[nz] = w[nz] / W[nz] / W[nz]
            w[~nz] = 0.
        return w

    def applyAinv(self, input_data, invPk0_grid=None, input_type='real', output_type='real'):
        """A^-1 = x invP / W^2 (base.py:364-389)."""
        assert input_type in ['fourier', 'real'], "Valid input types are 'fourier' and 'real' only!"
        assert output_type in ['fourier', 'real'], "Valid output types are 'fourier' and 'real' only!"
        x = self.to_fourier(input_data) if input_type == 'real' else input_data
        prec = nat.precision_of(x.dtype)
        rd = torch.float64 if prec == nat.PB_F64 else torch.float32
        if invPk0_grid is None:
            w = self.to_device_grid('ainv', self._ainv_weight, rd)
        else:
            wh = np.asarray(invPk0_grid, dtype=np.float64)
            if self.pixel_window != 'none':
                W = self.pixel_window_grid
                nz = W != 0
                wh = np.where(nz, wh / np.where(nz, W, 1.) / np.where(nz, W, 1.), 0.)
            w = torch.as_tensor(wh, dtype=rd, device=self.device)
        out = torch.empty_like(x)
        nat.spectral_filter(self.grid, prec, x.contiguous(), out, [(0, -1.0, np.inf, 0, 0, 1.0, 1)], w=w)
        if output_type == 'real':
            return self.to_real(out)
        return out
