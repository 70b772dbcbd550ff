"""ORACLE — test infrastructure only (the checker, never the product path).

A CPU FP64 restatement of PolyBin3D's binned polyspectrum hot path, written from the
reference's algorithm (file:line cited per function).  FFTs are scipy.fft in FP64 with
numpy's normalisation (forward unnormalised, inverse x 1/N^3), the convention of the
reference's `to_fourier`/`to_real` (base.py:176-229).  The O(N_bins N^3) real-space
triplet loop runs in plain C (oracle/oracle_loops.c) via ctypes.

Parity is pinned: tests/test_oracle_golden.py checks every function here against
fixtures produced by running the reference itself (tests/golden/make_golden.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import this.
"""
import ctypes
import os

import numpy as np
import scipy.fft
from scipy.interpolate import interp1d

_HERE = os.path.dirname(os.path.abspath(__file__))


# --------------------------------------------------------------------------------------
# C loops
# --------------------------------------------------------------------------------------
_loops = None


def _load_loops():
    global _loops
    if _loops is None:
        path = os.path.join(_HERE, "liboracle_loops.so")
        if not os.path.exists(path):
            build_loops()
        lib = ctypes.CDLL(path)
        P = ctypes.c_void_p
        I = ctypes.c_int64
        lib.oracle_triplet_sum.argtypes = [P, P, P, I, P, I, P, ctypes.c_int]
        lib.oracle_pair_sum.argtypes = [P, P, I, P, I, P, ctypes.c_int]
        _loops = lib
    return _loops


def build_loops():
    """Compile oracle/oracle_loops.c with gcc + OpenMP into oracle/liboracle_loops.so."""
    import subprocess
    src = os.path.join(_HERE, "oracle_loops.c")
    out = os.path.join(_HERE, "liboracle_loops.so")
    subprocess.check_call(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", src, "-o", out])
    return out


def triplet_sum(A, B, C, idx, nthreads=None):
    """out[t] = sum_x A[i1]B[i2]C[i3]; A,B,C are (n_maps, ...) float64 arrays.
    Restates assemble_b3 / sum_triplet (utils.pyx:614-636, 357-366)."""
    lib = _load_loops()
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    C = np.ascontiguousarray(C, dtype=np.float64)
    n_vox = int(np.prod(A.shape[1:]))
    idx = np.ascontiguousarray(idx, dtype=np.int64).reshape(-1, 3)
    out = np.zeros(len(idx), dtype=np.float64)
    lib.oracle_triplet_sum(A.ctypes.data, B.ctypes.data, C.ctypes.data, n_vox,
                           idx.ctypes.data, len(idx), out.ctypes.data,
                           int(nthreads or os.cpu_count()))
    return out


def pair_sum(A, B, idx, nthreads=None):
    """out[t] = sum_x A[i1]B[i2]  (sum_pair, utils.pyx:343-352)."""
    lib = _load_loops()
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    n_vox = int(np.prod(A.shape[1:]))
    idx = np.ascontiguousarray(idx, dtype=np.int64).reshape(-1, 2)
    out = np.zeros(len(idx), dtype=np.float64)
    lib.oracle_pair_sum(A.ctypes.data, B.ctypes.data, n_vox, idx.ctypes.data, len(idx),
                        out.ctypes.data, int(nthreads or os.cpu_count()))
    return out


# --------------------------------------------------------------------------------------
# small helpers
# --------------------------------------------------------------------------------------
def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 (Salmon et al., SC'11) on uint64 numpy arrays holding 32-bit words;
    returns the four output words.  Pinned to the published known-answer vectors in the
    CPU tests."""
    m32 = np.uint64(0xFFFFFFFF)
    M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
    c = [np.asarray(v, dtype=np.uint64) & m32 for v in (c0, c1, c2, c3)]
    k0, k1 = int(k0) & 0xFFFFFFFF, int(k1) & 0xFFFFFFFF
    for _ in range(10):
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        c = [(p1 >> np.uint64(32)) ^ c[1] ^ np.uint64(k0), p1 & m32, (p0 >> np.uint64(32)) ^ c[3] ^ np.uint64(k1),
             p0 & m32]
        k0 = (k0 + 0x9E3779B9) & 0xFFFFFFFF
        k1 = (k1 + 0xBB67AE85) & 0xFFFFFFFF
    return c


def legendre(l, mu):
    """Explicit Legendre polynomials, as utils.pyx:385-400."""
    if l == 0:
        return np.ones_like(mu)
    if l == 1:
        return mu
    if l == 2:
        return 0.5 * (3 * mu ** 2 - 1)
    if l == 3:
        return 0.5 * (5 * mu ** 3 - 3 * mu)
    if l == 4:
        return (35 * mu ** 4 - 30 * mu ** 2 + 3) / 8.0
    raise ValueError("l > 4 unsupported")


def real_harmonics_fourier(k_grids, lmax):
    """Real spherical harmonics of the unit vector, l = 1..4 (utils.pyx:518-609); the odd l
    are the reference's odd_l set."""
    kx, ky, kz = k_grids
    norm = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    safe = np.where(norm == 0, 1.0, norm)
    xh = np.where(norm == 0, 0.0, kx / safe)
    yh = np.where(norm == 0, 0.0, ky / safe)
    zh = np.where(norm == 0, 0.0, kz / safe)
    out = {}
    if lmax >= 1:
        out[1] = np.asarray([yh, zh, xh])
    if lmax >= 3:
        out[3] = np.asarray([
            (45.0 * xh ** 2 * yh - 15.0 * yh ** 3) * np.sqrt(1.0 / 360.0),
            (30.0 * xh * yh * zh) * np.sqrt(1.0 / 60.0),
            (-1.5 * xh ** 2 * yh - 1.5 * yh ** 3 + 6.0 * yh * zh ** 2) * np.sqrt(1.0 / 6.0),
            (-1.5 * xh ** 2 * zh - 1.5 * yh ** 2 * zh + zh ** 3),
            (-1.5 * xh ** 3 - 1.5 * xh * yh ** 2 + 6.0 * xh * zh ** 2) * np.sqrt(1.0 / 6.0),
            (15.0 * xh ** 2 * zh - 15.0 * yh ** 2 * zh) * np.sqrt(1.0 / 60.0),
            (15.0 * xh ** 3 - 45.0 * xh * yh ** 2) * np.sqrt(1.0 / 360.0)])
    if lmax >= 2:
        out[2] = np.asarray([
            6.0 * xh * yh * np.sqrt(1.0 / 12.0),
            3.0 * yh * zh * np.sqrt(1.0 / 3.0),
            zh ** 2 - xh ** 2 / 2.0 - yh ** 2 / 2.0,
            3.0 * xh * zh * np.sqrt(1.0 / 3.0),
            (3 * xh ** 2 - 3 * yh ** 2) * np.sqrt(1.0 / 12.0)])
    if lmax >= 4:
        out[4] = np.asarray([
            (420.0 * xh ** 3 * yh - 420.0 * xh * yh ** 3) * np.sqrt(1.0 / 20160.0),
            (315.0 * xh ** 2 * yh * zh - 105.0 * yh ** 3 * zh) * np.sqrt(1.0 / 2520.0),
            (-15.0 * xh ** 3 * yh - 15.0 * xh * yh ** 3 + 90.0 * xh * yh * zh ** 2) * np.sqrt(1.0 / 180.0),
            (-7.5 * xh ** 2 * yh * zh - 7.5 * yh ** 3 * zh + 10.0 * yh * zh ** 3) * np.sqrt(1.0 / 10.0),
            35.0 / 8.0 * zh ** 4 - 15.0 / 4.0 * zh ** 2 + 3.0 / 8.0,
            (-15.0 / 2.0 * xh ** 3 * zh - 15.0 * xh * yh ** 2 * zh / 2.0 + 10.0 * xh * zh ** 3) * np.sqrt(1.0 / 10.0),
            (-15.0 / 2.0 * xh ** 4 + 45.0 * xh ** 2 * zh ** 2 + 15.0 / 2.0 * yh ** 4 - 45.0 * yh ** 2 * zh ** 2) * np.sqrt(1.0 / 180.0),
            (105.0 * xh ** 3 * zh - 315.0 * xh * yh ** 2 * zh) * np.sqrt(1.0 / 2520.0),
            (105.0 * xh ** 4 - 630.0 * xh ** 2 * yh ** 2 + 105.0 * yh ** 4) * np.sqrt(1.0 / 20160.0)])
    return out


def pixel_window_1d(kind, x):
    """1-D voxel windows with first-order alias corrections (base.py:231-254); x = pi*n/N."""
    if kind == "cic":
        s = np.sin(x) ** 2.0
        return (1.0 - 2.0 / 3.0 * s) ** 0.5
    if kind == "tsc":
        s = np.sin(x) ** 2.0
        return (1.0 - s + 2.0 / 15 * s ** 2.0) ** 0.5
    if kind == "pcs":
        s = np.sin(x) ** 2.0
        return (1.0 - 4.0 / 3.0 * s + 2.0 / 5.0 * s ** 2 - 4.0 / 315.0 * s ** 3) ** 0.5
    if kind == "interlaced-cic":
        s = np.sinc(x / np.pi)
        v = np.ones_like(s)
        v[s != 0.0] = s[s != 0.0] ** 2.0
        return v
    if kind == "interlaced-tsc":
        return np.sinc(x / np.pi) ** 3.0
    if kind == "interlaced-pcs":
        return np.sinc(x / np.pi) ** 4.0
    raise ValueError(kind)


# --------------------------------------------------------------------------------------
# base geometry (base.py:20-144)
# --------------------------------------------------------------------------------------
class OracleBase:
    """Grids and FFTs of the reference base class, global sightline, real FFTs."""

    def __init__(self, boxsize, gridsize, Pk=None, pixel_window="none", nthreads=None, kernels=None,
                 boxcenter=None, sightline="global"):
        """kernels: optionally the reference's compiled Cython module (oracle/_ref, built from
        utils.pyx); its IntegrationUtils / MapUtils then run fourier_filter, cross_integrate,
        integrate_row and prod_real_diff (same results, multithreaded): the CPU-baseline
        timing mode.  Default: the numpy restatement."""
        self.boxsize = np.asarray(boxsize, dtype=np.float64)
        self.gridsize = np.asarray(gridsize, dtype=int)
        self.nthreads = nthreads or os.cpu_count()
        self.pixel_window = pixel_window
        self.sightline = sightline
        self.boxcenter = np.zeros(3) if boxcenter is None else np.asarray(boxcenter, dtype=np.float64)
        self.volume = self.boxsize.prod()
        self.kF = 2.0 * np.pi / self.boxsize                         # base.py:64
        self.kNy = self.gridsize * self.kF * 0.5                        # base.py:65
        if Pk is None:                                                  # base.py:68-70
            k_tmp = np.arange(0.0, np.max(self.kNy) * 2, np.min(self.kF) / 10.0)
            self.Pfid = np.asarray([k_tmp, 1.0 + 0.0 * k_tmp])
        else:
            self.Pfid = np.asarray(Pk)
        # fftshift order on axes 0,1; 0..N/2 on axis 2  (base.py:86-91)
        k_arrs = [np.fft.fftshift(np.arange(-self.gridsize[i] // 2, self.gridsize[i] // 2)) * self.kF[i]
                  for i in range(2)]
        k_arrs += [np.arange(0, self.gridsize[2] // 2 + 1) * self.kF[2]]
        self.k_arrs = k_arrs
        self.k_grids = np.meshgrid(*k_arrs, indexing="ij")
        self.modk_grid = np.sqrt(self.k_grids[0] ** 2 + self.k_grids[1] ** 2 + self.k_grids[2] ** 2)
        self.degeneracy_factor = np.asarray(1.0 + (self.k_grids[2] > 0), dtype=np.float64)   # base.py:94
        if pixel_window != "none":                                      # base.py:106-108
            w1d = [pixel_window_1d(pixel_window, np.pi / self.gridsize[i] * k_arrs[i] / self.kF[i])
                   for i in range(3)]
            self.pixel_window_grid = np.asarray(np.meshgrid(*w1d, indexing="ij")).prod(axis=0)
        self.muk_grid = np.zeros(self.modk_grid.shape)                  # base.py:115-116
        nz = self.modk_grid != 0
        if sightline == "global":                                       # base.py:111-114
            sv = np.asarray([0.0, 0.0, 1.0])
        else:
            sv = self.boxcenter / np.sqrt(np.sum(self.boxcenter ** 2))
        self.muk_grid[nz] = np.sum(sv[:, None] * np.asarray(self.k_grids)[:, nz], axis=0) / self.modk_grid[nz]
        self.Pk0_grid = interp1d(self.Pfid[0], self.Pfid[1], bounds_error=False,
                                 fill_value=0.0)(self.modk_grid)         # base.py:122
        self.invPk0_grid = np.zeros(self.modk_grid.shape)               # base.py:125-131
        good = (self.Pk0_grid != 0) & np.isfinite(self.Pk0_grid)
        self.invPk0_grid[good] = 1.0 / self.Pk0_grid[good]
        self.Pk0_grid[~np.isfinite(self.Pk0_grid)] = 0.0
        self.invPk0_grid[self.modk_grid == 0] = 1.0
        self.Pk0_grid[self.modk_grid == 0] = 1.0
        if sightline == "local":                                        # base.py:75-79
            r_arrs = [np.fft.fftshift(np.arange(-self.gridsize[i] // 2, self.gridsize[i] // 2)) * self.boxsize[i]
                      / self.gridsize[i] + self.boxcenter[i] for i in range(3)]
            self.r_grids = np.meshgrid(*r_arrs, indexing="ij")
        self._iu = self._mu = None
        if kernels is not None:                                         # base.py:138-144
            self._iu = kernels.IntegrationUtils(self.modk_grid, True, self.nthreads, self.degeneracy_factor,
                                                self.muk_grid)
            self._mu = kernels.MapUtils(self.modk_grid, self.gridsize, self.nthreads, self.muk_grid)

    # FFTs, numpy normalisation (base.py:176-229)
    def to_fourier(self, x):
        return scipy.fft.rfftn(np.asarray(x, dtype=np.float64), axes=(0, 1, 2), workers=self.nthreads)

    def to_real(self, k):
        return scipy.fft.irfftn(k, s=tuple(self.gridsize), axes=(0, 1, 2), workers=self.nthreads)

    # map utilities (utils.pyx:213-338)
    def in_bin(self, kmin, kmax):
        return (self.modk_grid >= kmin) & (self.modk_grid < kmax)

    def fourier_filter(self, kmap, l, kmin, kmax, l2=0):
        """Theta_b(k) L_l(mu) [L_l2(mu)] kmap  (fourier_filter / fourier_filter_ll, utils.pyx:283-320)."""
        if self._mu is not None and l2 == 0:
            return self._mu.fourier_filter(np.ascontiguousarray(kmap, dtype=np.complex128), l, kmin, kmax)
        out = np.zeros(self.modk_grid.shape, dtype=np.complex128)
        m = self.in_bin(kmin, kmax)
        leg = legendre(l, self.muk_grid[m]) * legendre(l2, self.muk_grid[m])
        out[m] = kmap[m] * leg
        return out

    def div_fourier(self, kmap, w):
        """kmap / w with 0 where w == 0 (utils.pyx:230-243)."""
        out = np.zeros_like(kmap, dtype=np.complex128)
        nz = w != 0
        out[nz] = kmap[nz] / w[nz]
        return out

    # k-bin reductions (utils.pyx:51-134); bins [k_b, k_b+1) with >= / <
    def integrate(self, spec, k_edges, l):
        vals = self.degeneracy_factor * (spec.real ** 2 + spec.imag ** 2) * legendre(l, self.muk_grid)
        return np.asarray([vals[self.in_bin(k_edges[b], k_edges[b + 1])].sum()
                           for b in range(len(k_edges) - 1)])

    def cross_integrate(self, s1, s2, k_edges, l):
        if self._iu is not None:
            return self._iu.cross_integrate(np.ascontiguousarray(s1), np.ascontiguousarray(s2),
                                            np.ascontiguousarray(k_edges, dtype=np.float64), l)
        vals = self.degeneracy_factor * (s1 * np.conj(s2)).real * legendre(l, self.muk_grid)
        return np.asarray([vals[self.in_bin(k_edges[b], k_edges[b + 1])].sum()
                           for b in range(len(k_edges) - 1)])

    def real_integrate_double(self, spec, l1, l2, k_edges):
        vals = self.degeneracy_factor * spec ** 2 * legendre(l1, self.muk_grid) * legendre(l2, self.muk_grid)
        return np.asarray([vals[self.in_bin(k_edges[b], k_edges[b + 1])].sum()
                           for b in range(len(k_edges) - 1)])

    def integrate_row(self, input_map, input_array, kmin, kmax):
        """out[j] = sum_{k in [kmin,kmax)} deg Re(conj(map) * array[j])  (utils.pyx:162-179)."""
        if self._iu is not None:
            return self._iu.integrate_row(np.ascontiguousarray(input_map), np.ascontiguousarray(input_array),
                                          kmin, kmax)
        m = self.in_bin(kmin, kmax)
        w = self.degeneracy_factor[m] * np.conj(input_map[m])
        return (input_array[:, m] * w[None, :]).real.sum(axis=1)

    def prod_real_diff(self, a, b, c, d):
        """a b - c d of real maps (prod_real_diff, utils.pyx:371-383)."""
        if self._mu is not None:
            return self._mu.prod_real_diff(a, b, c, d)
        return a * b - c * d

    # Gaussian random field from supplied white noise (base.py:305-353)
    def grf_from_noise(self, noise_re, noise_im, Pk_grid=None, include_pixel_window=True):
        """Reference draws noise_re, noise_im = np.random.randn(*N) twice after
        np.random.seed(seed) (base.py:315-316, 332); here they are inputs."""
        N = self.gridsize
        rand = noise_re + 1.0j * noise_im
        rand[0, 0, 0] = 0.0                                                     # base.py:333
        ii, jj, kk = np.meshgrid(*[np.arange(N[i]) for i in range(3)], indexing="ij")
        rand = 0.5 * (rand + np.conj(rand[(-ii) % N[0], (-jj) % N[1], (-kk) % N[2]]))  # 336-337
        rand = np.ascontiguousarray(rand[:, :, :N[2] // 2 + 1])                 # 340-341
        Pk_grid = self.Pk0_grid if Pk_grid is None else Pk_grid
        rand = rand * np.sqrt(Pk_grid) * N.prod() / np.sqrt(self.volume)        # 344
        if self.pixel_window != "none" and include_pixel_window:               # 347-348
            rand = rand * self.pixel_window_grid
        return rand

    def reference_noise(self, seed):
        """The reference's own draw: legacy MT19937 gaussians, real part first (base.py:316, 332)."""
        rs = np.random.RandomState(seed)
        re = rs.randn(*self.gridsize)
        im = rs.randn(*self.gridsize)
        return re, im

    def philox_noise(self, seed):
        """White noise of the on-device Philox GRF (not a reference function: the CUDA
        path's throughput mode draws its noise on the GPU).  Voxel p of the full grid:
        Box-Muller on the first two words of Philox4x32-10(counter=(p, 0x5A17, 0),
        key=seed)."""
        p = np.arange(int(np.prod(self.gridsize)), dtype=np.uint64)
        x = philox4x32_10(p & 0xFFFFFFFF, p >> np.uint64(32), np.full_like(p, 0x5A17), np.zeros_like(p),
                          int(seed) & 0xFFFFFFFF, (int(seed) >> 32) & 0xFFFFFFFF)
        u1 = (x[0].astype(np.float64) + 0.5) * 2.0 ** -32
        u2 = (x[1].astype(np.float64) + 0.5) * 2.0 ** -32
        rad = np.sqrt(-2.0 * np.log(u1))
        re = (rad * np.cos(2 * np.pi * u2)).reshape(tuple(self.gridsize))
        im = (rad * np.sin(2 * np.pi * u2)).reshape(tuple(self.gridsize))
        return re, im

    def apply_real_harmonics(self, a_fourier, l):
        """sum_m Y_lm(x) irfftn(Y_lm(k) a(k)) (base.py:391-400), even l."""
        yr = real_harmonics_fourier(self.r_grids, l)[l]
        yk = real_harmonics_fourier(self.k_grids, l)[l]
        out = np.zeros(tuple(self.gridsize))
        for m in range(len(yr)):
            out += self.to_real(a_fourier * yk[m]) * yr[m]
        return out

    def apply_fourier_harmonics(self, a_real, l):
        """sum_m Y_lm(k) rfftn(Y_lm(x) a(x)) (base.py:402-411) with the real harmonics of the
        positions and of the wavevectors (utils.pyx:518-609), even l."""
        yr = real_harmonics_fourier(self.r_grids, l)[l]
        yk = real_harmonics_fourier(self.k_grids, l)[l]
        out = np.zeros(self.modk_grid.shape, dtype=np.complex128)
        for m in range(len(yr)):
            out += self.to_fourier(a_real * yr[m]) * yk[m]
        return out

    def inverse_fiducial_draw(self):
        """The shot-noise GRFs' spectrum P_A = 1/P_fid on the grid, as generate_data
        interpolates it (zero outside the table), and 1/P_A extended by its end values
        (0 at k = 0)  (pspec.py:504-508)."""
        kP, PA = self.Pfid[0], 1.0 / self.Pfid[1]
        draw = interp1d(kP, PA, bounds_error=False, fill_value=0.0)(self.modk_grid)
        PA_grid = interp1d(kP, PA, bounds_error=False, fill_value=(PA[0], PA[-1]))(self.modk_grid)
        inv = np.zeros_like(PA_grid)
        nz = self.modk_grid != 0
        inv[nz] = 1.0 / PA_grid[nz]
        return draw, inv

    def applyAinv_fourier(self, a, invP=None):
        """A^-1 a = a invP (/W^2)  (base.py:364-389), Fourier in and out."""
        out = a * (self.invPk0_grid if invP is None else invP)
        if self.pixel_window != "none":
            out = self.div_fourier(self.div_fourier(out, self.pixel_window_grid), self.pixel_window_grid)
        return out


# --------------------------------------------------------------------------------------
# covariance filter (pspec.py:241-323, bspec.py:481-519, base.py:413-437)
# --------------------------------------------------------------------------------------
def xi_grids(b, Pk_cov):
    """Pk_grid of _compute_fisher (pspec.py:241-252, bspec.py:481-496): global, one grid
    P0(k) + L2(mu) P2(k) + L4(mu) P4(k); local, one grid per multipole.  Linear
    interpolation, zero outside the table."""
    from scipy.special import legendre as sp_legendre
    terms = [interp1d(Pk_cov[0], Pk_cov[i], bounds_error=False, fill_value=0.0)(b.modk_grid)
             for i in range(1, len(Pk_cov))]
    if b.sightline == "global":
        g = terms[0]
        for i, t in enumerate(terms[1:]):
            g = g + sp_legendre(2 * (i + 1))(b.muk_grid) * t
        return {0: g}
    return {2 * i: t for i, t in enumerate(terms)}


def apply_xi(b, X, x_real, xi, output):
    """apply_xi (base.py:413-437): P0 X, plus for the local sightline and each l > 0
    1/2 P_l sum_m Y_lm(k) FT[Y_lm(r) x] and 1/2 sum_m Y_lm(r) IFT[Y_lm(k) P_l X]."""
    PF = X * xi[0]
    if len(xi) == 1:
        return PF if output == "fourier" else b.to_real(PF)
    if x_real is None:
        raise ValueError("local multipoles of the covariance spectrum need the real-space map")
    PR = np.zeros(tuple(b.gridsize))
    for l in sorted(xi)[1:]:
        PF = PF + 0.5 * b.apply_fourier_harmonics(x_real, l) * xi[l]
        PR = PR + 0.5 * b.apply_real_harmonics(X * xi[l], l)
    return PF + b.to_fourier(PR) if output == "fourier" else b.to_real(PF) + PR


def trivial_sinv(b):
    """applySinv_trivial (base.py:355-362): the identity with real / Fourier conversion."""
    def f(x, input_type="real", output_type="real"):
        if input_type == output_type:
            return x
        return b.to_real(x) if input_type == "fourier" else b.to_fourier(x)
    return f


def cov_filter(b, x, real, xi, const_mask, mask_mean, point, mask_shot, sinv=None, sinv_t=None):
    """S^-1 [P xi P^dag + N] S^-dag x (pspec.py:277-290, 307-323; bspec.py:499-519); x is a
    real map if `real`, else a half spectrum; the output is a half spectrum.  point(x,
    transpose): the pointing matrix P or P^dag; sinv, sinv_t: S^-1 and S^-dag (default the
    trivial one)."""
    sinv = sinv or trivial_sinv(b)
    sinv_t = sinv_t or trivial_sinv(b)
    it = "real" if real else "fourier"
    if const_mask:
        Sid = sinv_t(x, it, "fourier")
        C = mask_mean ** 2 * apply_xi(b, Sid, None, xi, "fourier") + mask_mean * Sid
        return sinv(C, "fourier", "fourier")
    Sid = sinv_t(x, it, "real")
    Pd_real = point(Sid, True)
    C = apply_xi(b, b.to_fourier(Pd_real), Pd_real, xi, "real")
    return sinv(point(C, False) + mask_shot * Sid, "real", "fourier")


class Pointing:
    """The pointing matrix P of a varying mask (pspec.py:199-213, bspec.py:412-427): the mask,
    or with an integral constraint the mask times the map less its mean over mask_IC,
    globally (pointing_GIC, utils.pyx:405-424) or in radial shells of |r| (pointing_RIC,
    utils.pyx:448-481; voxels outside every shell give 0).  The transpose subtracts
    mask_IC times the mean of mask x map (utils.pyx:426-446, 483-516)."""

    def __init__(self, mask, mask_IC=None, kind="mask", radial_edges=None, modr=None):
        self.mask, self.mask_IC, self.kind = mask, mask_IC, kind
        if kind == "RIC":
            edges = np.asarray(radial_edges, dtype=np.float64)
            self.zidx = np.full(modr.shape, -1, dtype=np.int64)
            for iz in range(len(edges) - 1):
                self.zidx[(modr >= edges[iz]) & (modr < edges[iz + 1])] = iz
            self.nz = len(edges) - 1

    def __call__(self, x, transpose=False):
        if self.kind == "mask":
            return self.mask * x
        w = self.mask if transpose else self.mask_IC
        if self.kind == "GIC":
            av = np.sum(x * w) / np.sum(self.mask_IC)
            return self.mask * x - self.mask_IC * av if transpose else self.mask * (x - av)
        inz = self.zidx >= 0
        num = np.bincount(self.zidx[inz], weights=(x * w)[inz], minlength=self.nz)
        den = np.bincount(self.zidx[inz], weights=self.mask_IC[inz], minlength=self.nz)
        av = np.zeros(x.shape)
        av[inz] = (num / den)[self.zidx[inz]]
        out = self.mask * x - self.mask_IC * av if transpose else self.mask * (x - av)
        return np.where(inz, out, 0.0)


# --------------------------------------------------------------------------------------
# power spectrum (pspec.py)
# --------------------------------------------------------------------------------------
def _pointing_of(base, mask, mask_IC, add_GIC, add_RIC, radial_bins_RIC):
    """pspec.py:101-111, bspec.py:126-136: the RIC shells use |r| of the voxel positions."""
    if add_RIC:
        assert not add_GIC, "Radial integral constraint imposes global integral constraint automatically!"
        modr = np.sqrt(base.r_grids[0] ** 2 + base.r_grids[1] ** 2 + base.r_grids[2] ** 2)
        return Pointing(mask, np.asarray(mask_IC, dtype=np.float64), "RIC", radial_bins_RIC, modr)
    if add_GIC:
        return Pointing(mask, np.asarray(mask_IC, dtype=np.float64), "GIC")
    return Pointing(mask)


class OraclePSpec:
    def __init__(self, base, k_bins, lmax=2, mask=None, mask_IC=None, add_GIC=False, add_RIC=False,
                 radial_bins_RIC=None, odd_l=False, applySinv=None, applySinv_transpose=None):
        self.base = base
        # S^-1 and S^-dag (pspec.py:92-99): the trivial filter, or the caller's, whose
        # transpose defaults to itself
        self.sinv = applySinv or trivial_sinv(base)
        self.sinv_t = applySinv_transpose or (applySinv if applySinv is not None else trivial_sinv(base))
        self.k_bins = np.asarray(k_bins, dtype=np.float64)
        self.lmax = lmax
        self.odd_l = odd_l
        self.Nk = len(k_bins) - 1
        self.Nl = lmax + 1 if odd_l else lmax // 2 + 1               # pspec.py:37-39
        self.Nl_even = lmax // 2 + 1
        self.N_bins = self.Nk * self.Nl
        if mask is None:                                             # pspec.py:62-81
            self.const_mask, self.mask_mean, self.sq_mask_mean = True, 1.0, 1.0
        else:
            self.mask = np.asarray(mask, dtype=np.float64)
            if np.std(self.mask) < 1e-12:
                self.const_mask = True
                self.mask_mean = np.mean(self.mask)
            else:
                self.const_mask = False
            self.sq_mask_mean = np.mean(self.mask ** 2)
            self.point = _pointing_of(base, self.mask, mask_IC, add_GIC, add_RIC, radial_bins_RIC)

    def ell(self, li):
        """Multipole of block li: 2 li, or li with odd_l (pspec.py:667)."""
        return li * (2 - self.odd_l)

    def numerator(self, data, filtering="ideal"):
        """_compute_pk_numerator (pspec.py:613-686); trivial S^-1.  The ideal numerator has
        the even multipoles only; with odd_l the S^-1 one has l = 0..lmax, the odd blocks
        crossed with -i H_l[x] so that they are real (pspec.py:674-676)."""
        b = self.base
        data = np.asarray(data, dtype=np.float64)
        x = b.to_fourier(data)
        if b.pixel_window != "none":
            x = b.div_fourier(x, b.pixel_window_grid)
        if filtering == "ideal":
            x = x * b.invPk0_grid / np.sqrt(self.sq_mask_mean)
        elif b.pixel_window != "none":                                   # pspec.py:629-640
            x = self.sinv(x, "fourier", "fourier")
        else:
            x = self.sinv(data, "real", "fourier")
        Nl = self.Nl if filtering != "ideal" else self.Nl_even
        odd = self.odd_l and filtering != "ideal"
        out = np.zeros(Nl * self.Nk)
        for li in range(Nl):
            l = li * (2 - odd)
            if b.sightline == "global" or li == 0:
                out[li * self.Nk:(li + 1) * self.Nk] = 0.5 * b.integrate(x, self.k_bins, l)
            else:                                                        # pspec.py:672-680
                lm = b.apply_fourier_harmonics(b.to_real(x), l)
                if l % 2 == 1:
                    lm = -1.0j * lm
                out[li * self.Nk:(li + 1) * self.Nk] = 0.5 * b.cross_integrate(x, lm, self.k_bins, 0)
        return out * b.volume / b.gridsize.prod() ** 2

    def fisher_ideal(self, discreteness_correction=True):
        """compute_fisher_ideal with the base fiducial spectrum (pspec.py:702-752)."""
        b = self.base
        nb = self.Nl_even * self.Nk
        fish = np.zeros((nb, nb))
        if discreteness_correction:
            for la in range(self.Nl_even):
                for lb in range(self.Nl_even):
                    fish[la * self.Nk:(la + 1) * self.Nk, lb * self.Nk:(lb + 1) * self.Nk] = np.diag(
                        0.5 * b.real_integrate_double(b.invPk0_grid, 2 * la, 2 * lb, self.k_bins))
        else:
            d = 0.5 * b.real_integrate_double(b.invPk0_grid, 0, 0, self.k_bins)
            for la in range(self.Nl_even):
                fish[la * self.Nk:(la + 1) * self.Nk, la * self.Nk:(la + 1) * self.Nk] = np.diag(d) / (4.0 * la + 1.0)
        return fish

    def Pk_ideal(self, data, fish=None):
        fish = self.fisher_ideal() if fish is None else fish
        out = np.linalg.inv(fish) @ self.numerator(data, "ideal")      # pspec.py:775
        return {"p%d" % (2 * li): out[li * self.Nk:(li + 1) * self.Nk] for li in range(self.Nl_even)}

    def fisher_contribution(self, noise_pair):
        """_compute_fisher, no covariance, no theory, trivial S^-1 (pspec.py:215-493)."""
        return self._contribution(noise_pair)

    def covariance_contribution(self, noise_pair, Pk_cov, mask_shot=None):
        """compute_covariance_contribution (pspec.py:149-162): the Fisher rows with the
        filter S^-1 P replaced by S^-1 [P xi P^dag + N] S^-dag, xi the correlation of the
        spectrum Pk_cov = [k, P0(, P2(, P4))] and N the shot mask (the mask mean for a
        constant mask)."""
        assert len(np.asarray(Pk_cov).shape) == 2 and len(Pk_cov) in (2, 3, 4)
        assert (len(Pk_cov) - 2) * 2 <= self.lmax
        return self._contribution(noise_pair, xi=self.xi_grids(Pk_cov), mask_shot=mask_shot)

    def theory_contribution(self, noise_pair, k_bins_theory, lmax_theory=None, include_wideangle=False):
        """compute_theory_contribution (pspec.py:164-196): the Fisher contribution and the
        rectangular binning matrix whose column block l_t holds the cross integrals of each
        Q-map with A^-1 a (global: weighted by L_l_t(mu); local: with
        sum_m Y_lm(k) FT[Y_lm(r) A^-1 a]) in the theory k-bins; with include_wideangle the
        odd-l terms of A^-1 a / |r| add to the l = 2, 4 blocks (pspec.py:424-438)."""
        k_th = np.asarray(k_bins_theory, dtype=np.float64)
        lt = self.lmax if lmax_theory is None else lmax_theory
        odd_t = True if include_wideangle else self.odd_l
        nlt = lt + 1 if (odd_t and not include_wideangle) else lt // 2 + 1     # pspec.py:222-228
        return self._contribution(noise_pair, theory=(k_th, nlt, lt, include_wideangle, odd_t))

    def xi_grids(self, Pk_cov):
        return xi_grids(self.base, Pk_cov)

    def cov_filter(self, x, real, xi, mask_shot):
        return cov_filter(self.base, x, real, xi, self.const_mask, getattr(self, "mask_mean", None),
                          None if self.const_mask else self.point, mask_shot, self.sinv, self.sinv_t)

    def _contribution(self, noise_pair, xi=None, mask_shot=None, theory=None):
        """_compute_fisher, global and local (even l) sightlines (pspec.py:215-493)."""
        b = self.base
        a = b.grf_from_noise(*noise_pair)                                # pspec.py:266
        if not self.const_mask:
            a_real = b.to_real(a)                                        # 268
        Ainv = b.applyAinv_fourier(a)                                    # 328

        def dagger(x, real):                                             # 291-323
            if xi is not None:
                return self.cov_filter(x, real, xi, mask_shot)
            it = "real" if real else "fourier"
            if self.const_mask:
                return self.mask_mean * self.sinv_t(x, it, "fourier")
            return b.to_fourier(self.point(self.sinv_t(x, it, "real"), True))

        if xi is not None:                                               # 270-290, 330-332
            SinvP = dagger(a, False) if self.const_mask else dagger(a_real, True)
        elif self.const_mask:                                            # 273-276
            SinvP = self.mask_mean * self.sinv(a, "fourier", "fourier")
        else:
            SinvP = self.sinv(self.point(a_real, False), "real", "fourier")
        fish = np.zeros((self.N_bins, self.N_bins))
        bm = None if theory is None else np.zeros((self.N_bins, theory[1] * (len(theory[0]) - 1)))
        scaling = 0.5 * b.volume / b.gridsize.prod() ** 2                # 390
        if b.sightline == "local":
            self._fisher_local(Ainv, SinvP, scaling, dagger, fish, theory, bm)
            return fish if theory is None else (fish, bm)
        for li in range(self.Nl):
            for ki in range(self.Nk):
                Q = dagger(b.fourier_filter(SinvP, 2 * li, self.k_bins[ki], self.k_bins[ki + 1]), False)
                row = li * self.Nk + ki
                for lp in range(self.Nl):                                # 394-401
                    fish[row, lp * self.Nk:(lp + 1) * self.Nk] += scaling * b.cross_integrate(
                        Ainv, Q, self.k_bins, 2 * lp)
                if theory is not None:                                   # 395-402
                    kt, nlt = theory[:2]
                    nkt = len(kt) - 1
                    for lt in range(nlt):
                        bm[row, lt * nkt:(lt + 1) * nkt] += scaling * b.cross_integrate(Ainv, Q, kt, 2 * lt)
        return fish if theory is None else (fish, bm)

    @staticmethod
    def derivative_coefficient(k):
        """Coefficients of the numerical k dP/dk in the theory bins (pspec.py:368-378)."""
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

    def _fisher_local(self, Ainv, SinvP, scaling, dagger, fish, theory=None, bm=None):
        """_compute_fisher, local sightline (pspec.py:334-366, 380-438, 456-486).
        Monopole rows Q = D Theta_b SinvP; multipole rows
        Q = 1/2 D Theta_b H_l[SinvP] + 1/2 D sum_m Y_lm(r) IFT[Theta_b Y_lm(k) SinvP]
        (odd l: both parts times -i) with D = (S^-1 P)^dag (or its covariance form) and
        H_l[x] = sum_m Y_lm(k) FT[Y_lm(r) IFT x]; the row against column block l is the
        cross integral of Q (odd l: i Q) with A^-1 a (l = 0) or with H_l[A^-1 a], in the data
        bins and, for the theory matrix, the theory bins.  Wide-angle theory terms: the odd
        l maps H_l[A^-1 a / |r|] enter the l = 2, 4 blocks with the complex per-bin
        coefficients of pspec.py:424-438."""
        b = self.base
        A_real = b.to_real(Ainv)
        legA = {}

        def leg(l, src="A"):
            key = (l, src)
            if key not in legA:
                if src == "A":
                    x = A_real
                else:                                                    # div_real, utils.pyx:265-278
                    r = np.sqrt(b.r_grids[0] ** 2 + b.r_grids[1] ** 2 + b.r_grids[2] ** 2)
                    x = np.where(r != 0, A_real / np.where(r != 0, r, 1.0), 0.0)
                legA[key] = b.apply_fourier_harmonics(x, l)
            return legA[key]

        SinvP_real = b.to_real(SinvP)

        def add(row, Q):                                                 # 380-438
            fish[row, :self.Nk] += scaling * b.cross_integrate(Ainv, Q, self.k_bins, 0)
            for li in range(1, self.Nl):
                l = self.ell(li)
                fish[row, li * self.Nk:(li + 1) * self.Nk] += scaling * b.cross_integrate(
                    leg(l), 1.0j * Q if l % 2 else Q, self.k_bins, 0)
            if theory is None:
                return
            kt, nlt, lt, wide, odd_t = theory
            nkt = len(kt) - 1
            bm[row, :nkt] += scaling * b.cross_integrate(Ainv, Q, kt, 0)
            if not wide:
                for li in range(1, nlt):
                    l = li * (2 - odd_t)
                    bm[row, li * nkt:(li + 1) * nkt] += scaling * b.cross_integrate(
                        leg(l), 1.0j * Q if l % 2 else Q, kt, 0)
                return
            kfac = self.derivative_coefficient(kt)
            for l in range(1, lt + 1):
                if l % 2 == 0:
                    bm[row, l // 2 * nkt:(l // 2 + 1) * nkt] += scaling * b.cross_integrate(leg(l), Q, kt, 0)
                    continue
                terms = []
                if l == 1 and lt >= 2:
                    terms.append((1, 3.0j / 5.0 * (3 + kfac)))
                if l == 3 and lt >= 2:
                    terms.append((1, 3.0j / 5.0 * (2 - kfac)))
                if l == 3 and lt >= 4:
                    terms.append((2, 10.0j / 9.0 * (5 + kfac)))
                for blk, coeff in terms:                                 # utils.pyx:139-157
                    bm[row, blk * nkt:(blk + 1) * nkt] += scaling * self.cross_wcoeff(coeff, leg(l, "A/r"), Q, kt)

        for ki in range(self.Nk):                                        # 442-445
            add(ki, dagger(b.fourier_filter(SinvP, 0, self.k_bins[ki], self.k_bins[ki + 1]), False))
        for li in range(1, self.Nl):                                     # 456-486
            l = self.ell(li)
            ph = -1.0j if l % 2 else 1.0
            lg = b.apply_fourier_harmonics(SinvP_real, l)
            yr = real_harmonics_fourier(b.r_grids, l)[l]
            yk = real_harmonics_fourier(b.k_grids, l)[l]
            for ki in range(self.Nk):
                Q = 0.5 * dagger(ph * b.fourier_filter(lg, 0, self.k_bins[ki], self.k_bins[ki + 1]), False)
                real_map = np.zeros(tuple(b.gridsize))
                m = b.in_bin(self.k_bins[ki], self.k_bins[ki + 1])
                for mi in range(len(yr)):
                    km = np.zeros(b.modk_grid.shape, dtype=np.complex128)
                    km[m] = SinvP[m] * yk[mi][m]
                    real_map += b.to_real(ph * km) * yr[mi]
                Q = Q + 0.5 * dagger(real_map, True)
                add(li * self.Nk + ki, Q)
        return fish

    def cross_wcoeff(self, coeff, s1, s2, k_edges):
        """cross_integrate_wcoeff (utils.pyx:139-157): sum deg Re(c_b s1 conj(s2)) per bin."""
        b = self.base
        out = np.zeros(len(k_edges) - 1)
        for i in range(len(out)):
            m = b.in_bin(k_edges[i], k_edges[i + 1])
            out[i] = np.sum(b.degeneracy_factor[m] * (coeff[i] * s1[m] * np.conj(s2[m])).real)
        return out

    def shot_contribution(self, noise_pair, mask_shot=None):
        """compute_shot_contribution, global sightline (pspec.py:495-549): a = GRF of
        P_A = 1/P_fid (pixel window included), S^-1 N A^-1 a with A^-1 = (1/P_A)/W^2 and N the
        shot mask, then half the cross integral of S^-1 a with it."""
        b = self.base
        draw, invPA = b.inverse_fiducial_draw()
        a = b.grf_from_noise(*noise_pair, Pk_grid=draw)                  # 511
        if self.const_mask:                                              # 514-519
            sna = self.mask_mean * self.sinv(b.applyAinv_fourier(a, invPA), "fourier", "fourier")
        else:
            sna = self.sinv(b.to_real(b.applyAinv_fourier(a, invPA)) * mask_shot, "real", "fourier")
        a = self.sinv(a, "fourier", "fourier")                           # 522
        shot = np.zeros(self.N_bins)
        for li in range(self.Nl):                                        # 526-544
            if b.sightline == "global" or li == 0:
                shot[li * self.Nk:(li + 1) * self.Nk] = 0.5 * b.cross_integrate(a, sna, self.k_bins, 2 * li)
            else:                                                        # 535-544
                l = self.ell(li)
                lm = b.apply_fourier_harmonics(b.to_real(a), l)
                if l % 2:
                    lm = -1.0j * lm
                shot[li * self.Nk:(li + 1) * self.Nk] = 0.5 * b.cross_integrate(lm, sna, self.k_bins, 0)
        return shot * b.volume / b.gridsize.prod() ** 2


# --------------------------------------------------------------------------------------
# bispectrum (bspec.py)
# --------------------------------------------------------------------------------------
def check_bin(k_bins, k_bins_squeeze, b1, b2, b3, include_partial_triangles=False):
    """Triangle test on bin centres, or on bin edges for partial triangles (bspec.py:171-199)."""
    ks = k_bins_squeeze
    if include_partial_triangles:
        k3_hi = ks[b1 + 1] + ks[b2 + 1]
        if b1 > b2:
            k3_lo = ks[b1] - ks[b2 + 1]
        elif b1 == b2:
            k3_lo = 0.0
        else:
            k3_lo = ks[b2] - ks[b1 + 1]
        return not (ks[b3] >= k3_hi - 1e-10 or ks[b3 + 1] <= k3_lo + 1e-10)
    k1 = 0.5 * (k_bins[b1] + k_bins[b1 + 1])
    k2 = 0.5 * (ks[b2] + ks[b2 + 1])
    k3 = 0.5 * (ks[b3] + ks[b3 + 1])
    return not (k3 < abs(k1 - k2) or k3 > k1 + k2)


def all_bins_list(k_bins, lmax, k_bins_squeeze=None, include_partial_triangles=False):
    """(b1,b2,b3,l) rows, l outer, b1<=b2<=b3 (bspec.py:67-75)."""
    k_bins = np.asarray(k_bins)
    ks = k_bins if k_bins_squeeze is None else np.asarray(k_bins_squeeze)
    Nk, Nks = len(k_bins) - 1, len(ks) - 1
    rows = []
    for l in range(0, lmax + 1, 2):
        for b1 in range(Nk):
            for b2 in range(b1, Nks):
                for b3 in range(b2, Nks):
                    if check_bin(k_bins, ks, b1, b2, b3, include_partial_triangles):
                        rows.append((b1, b2, b3, l))
    return np.asarray(rows, dtype=np.int64)


class OracleBSpec:
    def __init__(self, base, k_bins, lmax=0, mask=None, k_bins_squeeze=None,
                 include_partial_triangles=False, mask_IC=None, add_GIC=False, add_RIC=False,
                 radial_bins_RIC=None, applySinv=None, applySinv_transpose=None):
        self.base = base
        # S^-1 and S^-dag (bspec.py:117-124)
        self.sinv = applySinv or trivial_sinv(base)
        self.sinv_t = applySinv_transpose or (applySinv if applySinv is not None else trivial_sinv(base))
        self.k_bins = np.asarray(k_bins, dtype=np.float64)
        self.k_bins_squeeze = self.k_bins.copy() if k_bins_squeeze is None else np.asarray(k_bins_squeeze, dtype=np.float64)
        self.lmax = lmax
        self.Nk = len(self.k_bins) - 1
        self.Nk_squeeze = len(self.k_bins_squeeze) - 1
        self.Nl = lmax // 2 + 1
        self.all_bins = all_bins_list(self.k_bins, lmax, self.k_bins_squeeze, include_partial_triangles)
        self.N_bins = len(self.all_bins)
        self.N3 = self.N_bins // self.Nl
        if mask is None:                                                 # bspec.py:87-106
            self.const_mask, self.mask_mean, self.cube_mask_mean = True, 1.0, 1.0
        else:
            self.mask = np.asarray(mask, dtype=np.float64)
            if np.std(self.mask) < 1e-12:
                self.const_mask = True
                self.mask_mean = np.mean(self.mask)
            else:
                self.const_mask = False
            self.cube_mask_mean = np.mean(self.mask ** 3)
            self.point = _pointing_of(base, self.mask, mask_IC, add_GIC, add_RIC, radial_bins_RIC)
        # Pk_fid=None: unit weighting on k >= kF/10 grid (bspec.py:139-153)
        b = base
        k_tmp = np.arange(np.min(b.kF) / 10.0, np.max(b.kNy) * 2, np.min(b.kF) / 10.0)
        P = interp1d(k_tmp, 1.0 + 0.0 * k_tmp, bounds_error=False, fill_value=0.0)(b.modk_grid)
        self.invPk0 = np.zeros(P.shape)
        self.invPk0[P != 0] = 1.0 / P[P != 0]

    def triplet_index(self):
        """Map-index triplets for assemble_b3 over maps ordered (l/2, b)."""
        nb = self.Nk_squeeze
        ab = self.all_bins
        return np.stack([ab[:, 0], ab[:, 1], (ab[:, 3] // 2) * nb + ab[:, 2]], axis=1)

    def symmetry_factor(self):
        """_compute_symmetry_factor (bspec.py:222-279)."""
        b = self.base
        sym = []
        for (b1, b2, b3, l) in self.all_bins[self.all_bins[:, 3] == 0]:
            if b1 == b2 and b1 == b3:
                sym.append(6.0)
            elif b1 == b2 or b1 == b3 or b2 == b3:
                sym.append(2.0)
            else:
                sym.append(1.0)
        if self.lmax > 0:
            ks = self.k_bins_squeeze
            invP = self.invPk0.astype(np.complex128)
            bins = np.asarray([b.to_real(b.fourier_filter(invP, 0, ks[i], ks[i + 1]))
                               for i in range(self.Nk_squeeze)])
            ylm = real_harmonics_fourier(b.k_grids, self.lmax)
            for l in range(2, self.lmax + 1, 2):
                bin23 = np.zeros_like(bins)
                for i in range(self.Nk_squeeze):
                    m = b.in_bin(ks[i], ks[i + 1])
                    for y in ylm[l]:
                        km = np.zeros(b.modk_grid.shape, dtype=np.complex128)
                        km[m] = invP[m] * y[m]
                        bin23[i] += b.to_real(km) ** 2
                for (b1, b2, b3, ll) in self.all_bins[self.all_bins[:, 3] == l]:
                    if b1 != b2 and b2 != b3:
                        sym.append(1.0)
                    elif b1 == b2 and b2 != b3:
                        sym.append(2.0)
                    elif b1 != b2 and b2 == b3:
                        sym.append(1.0 + np.sum(bins[b1] * bin23[b3]) / np.sum(bins[b1] * bins[b3] * bins[b3]))
                    else:
                        sym.append(2.0 * (1.0 + 2.0 * np.sum(bins[b3] * bin23[b3]) / np.sum(bins[b3] ** 3)))
        return np.asarray(sym)

    def g_maps(self, weighted_fourier):
        """g[l/2, b] = irfftn(Theta_b L_l x)  (bspec.py:936-956)."""
        b = self.base
        ks = self.k_bins_squeeze
        g = np.zeros((self.Nl, self.Nk_squeeze) + tuple(b.gridsize))
        real = b.to_real(weighted_fourier) if (b.sightline == "local" and self.lmax > 0) else None
        for l in range(0, self.lmax + 1, 2):
            if l > 0 and b.sightline == "local":                        # bspec.py:950-954
                src, ll = b.apply_fourier_harmonics(real, l), 0
            else:
                src, ll = weighted_fourier, l
            for i in range(self.Nk_squeeze):
                g[l // 2, i] = b.to_real(b.fourier_filter(src, ll, ks[i], ks[i + 1]))
        return g

    def weighted_data(self, data, filtering="ideal"):
        """S^-1 d in Fourier space (bspec.py:912-929)."""
        b = self.base
        data = np.asarray(data, dtype=np.float64)
        x = b.to_fourier(data)
        if b.pixel_window != "none":
            x = b.div_fourier(x, b.pixel_window_grid)
        if filtering == "ideal":
            return x * self.invPk0 / self.cube_mask_mean ** (1.0 / 3.0)
        if b.pixel_window != "none":
            return self.sinv(x, "fourier", "fourier")
        return self.sinv(data, "real", "fourier")

    def numerator(self, data, filtering="ideal", sym=None, sims=None):
        """_compute_bk_numerator (bspec.py:895-983); with `sims` (a list of bias-simulation
        spectra from sim_spectrum / generated_sim) the linear term is included."""
        b = self.base
        sym = self.symmetry_factor() if sym is None else sym
        g = self.g_maps(self.weighted_data(data, filtering))
        flat = g.reshape(self.Nl * self.Nk_squeeze, -1)
        B3 = triplet_sum(flat, flat, flat, self.triplet_index(), b.nthreads)
        if sims is not None:
            B3 = B3 + self.linear_term(g, sims)
        return B3 * b.volume / b.gridsize.prod() / sym

    def bshot_sum(self, A, B, C):
        """assemble_bshot (utils.pyx:641-663): the triplet sums of all six orderings of the
        map sets A, B, C over (b1, b2, (l, b3))."""
        n = self.Nl * self.Nk_squeeze
        f = [np.asarray(M).reshape(n, -1) for M in (A, B, C)]
        idx = self.triplet_index()
        out = np.zeros(len(idx))
        for (i, j, k) in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
            out += triplet_sum(f[i], f[j], f[k], idx, self.base.nthreads)
        return out

    def shot_contribution(self, noise1, noise2, mask_shot, data=None, data2=None, sym=None, cubic_only=False):
        """compute_shot_contribution, global sightline (bspec.py:695-861).  Two GRFs of
        P_A = 1/P_fid with the pixel window; A^-1 = P_fid / W^2 (the base grid, 772); maps
        A, B of S^-1 a1, S^-1 a2 (no window division), C of the shot-masked product
        (A^-1 a1)(A^-1 a2), D, E of (A^-1 a_i) d2; cubic = bshot(A, B, C) V/(6 N^3 sym),
        quadratic = (bshot(g, A, D) + bshot(g, B, E)) V/(4 N^3 sym); returns quadratic - 2 cubic."""
        b = self.base
        sym = self.symmetry_factor() if sym is None else sym
        draw, _ = b.inverse_fiducial_draw()
        a1 = b.grf_from_noise(*noise1, Pk_grid=draw)                     # 775-776
        a2 = b.grf_from_noise(*noise2, Pk_grid=draw)
        r1 = b.to_real(b.applyAinv_fourier(a1, b.Pk0_grid))              # 779-780
        r2 = b.to_real(b.applyAinv_fourier(a2, b.Pk0_grid))
        gA = self.g_maps(self.sinv(a1, "fourier", "fourier"))          # 788-790
        gB = self.g_maps(self.sinv(a2, "fourier", "fourier"))
        gC = self.g_maps(self.sinv(r1 * r2 * mask_shot, "real", "fourier"))   # 781
        norm = b.volume / b.gridsize.prod() / sym
        cubic = self.bshot_sum(gA, gB, gC) * norm / 6.0                  # 849-850
        if cubic_only:
            return cubic
        g = self.g_maps(self.weighted_data(data, "Sinv"))               # 730-768
        gD = self.g_maps(self.sinv(r1 * data2, "real", "fourier"))      # 783-784
        gE = self.g_maps(self.sinv(r2 * data2, "real", "fourier"))
        quad = 0.5 * (self.bshot_sum(g, gA, gD) + self.bshot_sum(g, gB, gE)) * norm / 2.0   # 853-856
        return quad - 2.0 * cubic

    # bias simulations for the linear term (bspec.py:281-410)
    def sim_spectrum(self, sim, input_type="real"):
        """_process_sim before the g-maps (bspec.py:288-300): S^-1 of one simulation in
        Fourier space, the pixel window divided out first when there is one."""
        b = self.base
        if b.pixel_window == "none":
            return self.sinv(sim, input_type, "fourier")
        if input_type == "real":
            x = b.to_fourier(np.asarray(sim, dtype=np.float64))
        else:
            x = np.array(sim, dtype=np.complex128)
        return self.sinv(x / b.pixel_window_grid, "fourier", "fourier")

    def generated_sim(self, ii, Pk_grid=None):
        """load_sim_data of generate_sims (bspec.py:377-392): the GRF of seed 1e5 + ii, times
        the mask mean (constant mask) or through the mask in real space."""
        b = self.base
        re, im = b.reference_noise(int(1e5) + ii)
        if self.const_mask:
            return self.sim_spectrum(self.mask_mean * b.grf_from_noise(re, im, Pk_grid), "fourier")
        s = self.point(b.to_real(b.grf_from_noise(re, im, Pk_grid, include_pixel_window=False)))
        if b.pixel_window != "none":
            return self.sim_spectrum(b.to_fourier(s) * b.pixel_window_grid, "fourier")
        return self.sim_spectrum(s, "real")

    def linear_term(self, g, sims):
        """B1 = -1/N_it sum_ii assemble_b1(g, g_ii) (bspec.py:963-978), where
        assemble_b1 sums g[0,b1] s[0,b2] s[l/2,b3] + s[0,b1] g[0,b2] s[l/2,b3]
        + s[0,b1] s[0,b2] g[l/2,b3] over voxels (utils.pyx:668-692)."""
        n = self.Nl * self.Nk_squeeze
        flat = g.reshape(n, -1)
        idx = self.triplet_index()
        out = np.zeros(len(idx))
        for xs in sims:
            s = self.g_maps(xs).reshape(n, -1)
            out += (triplet_sum(flat, s, s, idx, self.base.nthreads) + triplet_sum(s, flat, s, idx, self.base.nthreads)
                    + triplet_sum(s, s, flat, idx, self.base.nthreads))
        return -out / len(sims)

    def fisher_ideal(self, discreteness_correction=True, sym=None):
        """compute_fisher_ideal (bspec.py:999-1083)."""
        b = self.base
        sym = self.symmetry_factor() if sym is None else sym
        ks = self.k_bins_squeeze
        invP = self.invPk0.astype(np.complex128)
        nb = self.Nk_squeeze
        ab = self.all_bins[:self.N3, :3]
        if discreteness_correction:
            fish = np.zeros((self.N_bins, self.N_bins))
            u = np.asarray([[b.to_real(b.fourier_filter(invP, l, ks[i], ks[i + 1])) for i in range(nb)]
                            for l in range(0, self.lmax + 1, 2)])
            for l in range(0, self.lmax + 1, 2):
                for lp in range(l, self.lmax + 1, 2):
                    ull = np.asarray([b.to_real(b.fourier_filter(invP, l, ks[i], ks[i + 1], l2=lp))
                                      for i in range(nb)])
                    T1 = triplet_sum(u[0], u[0], ull, ab, b.nthreads)
                    T2 = triplet_sum(u[0], u[l // 2], u[lp // 2], ab, b.nthreads)
                    for i in range(self.N3):
                        b1, b2, b3 = ab[i]
                        if b1 != b2 and b2 != b3:
                            v = T1[i]
                        elif b1 == b2 and b2 != b3:
                            v = 2.0 * T1[i]
                        elif b1 != b2 and b2 == b3:
                            v = T2[i] + T1[i]
                        else:
                            v = 4.0 * T2[i] + 2.0 * T1[i]
                        fish[l // 2 * self.N3 + i, lp // 2 * self.N3 + i] = v
            fish = fish + fish.T - np.diag(np.diag(fish))
            fish = fish / np.outer(sym, sym) * b.gridsize.prod() ** 2 / b.volume
        else:
            u0 = np.asarray([b.to_real(b.fourier_filter(invP, 0, ks[i], ks[i + 1])) for i in range(nb)])
            Ntri = triplet_sum(u0, u0, u0, ab, b.nthreads)
            d = np.concatenate([Ntri / (2.0 * l + 1.0) for l in range(0, self.lmax + 1, 2)])
            fish = np.diag(d / sym) * b.gridsize.prod() ** 2 / b.volume
        return fish

    def Bk_ideal(self, data, fish=None, sym=None):
        sym = self.symmetry_factor() if sym is None else sym
        fish = self.fisher_ideal(sym=sym) if fish is None else fish
        out = np.linalg.inv(fish) @ self.numerator(data, "ideal", sym=sym)   # bspec.py:1110
        return {"b%d" % l: out[l // 2 * self.N3:(l // 2 + 1) * self.N3] for l in range(0, self.lmax + 1, 2)}

    def covariance_contribution(self, noise1, noise2, Pk_cov, mask_shot_2pt=None, sym=None):
        """compute_covariance_contribution (bspec.py:447-471): the Fisher contribution with
        S^-1 P replaced by S^-1 [P xi P^dag + N] S^-dag, N the two-point shot mask."""
        assert len(np.asarray(Pk_cov).shape) == 2 and len(Pk_cov) in (2, 3, 4)
        return self.fisher_contribution(noise1, noise2, sym=sym, xi=xi_grids(self.base, Pk_cov),
                                        mask_shot=mask_shot_2pt)

    def fisher_contribution(self, noise1, noise2, sym=None, return_Q=False, xi=None, mask_shot=None):
        """_compute_fisher, trivial S^-1 (bspec.py:473-676); for the local sightline the
        l > 0 maps come from the harmonic transform of each weighted map (548-577) and the
        l leg of the A^-1 Q maps is applied in real space (621-631).  With xi, the
        covariance form of the filter (499-519)."""
        b = self.base
        sym = self.symmetry_factor() if sym is None else sym
        ks = self.k_bins_squeeze
        ab = self.all_bins
        nks = self.Nk_squeeze
        a1 = b.grf_from_noise(*noise1)                                   # 648-649
        a2 = b.grf_from_noise(*noise2)
        if not self.const_mask:
            ar1, ar2 = b.to_real(a1), b.to_real(a2)                      # 651-653

        def apply_filter(x_fourier=None, x_real=None):                   # 499-519
            if xi is not None:
                return cov_filter(b, x_fourier if self.const_mask else x_real, not self.const_mask, xi,
                                  self.const_mask, getattr(self, "mask_mean", None),
                                  None if self.const_mask else self.point, mask_shot, self.sinv, self.sinv_t)
            if self.const_mask:
                return self.mask_mean * self.sinv(x_fourier, "fourier", "fourier")
            return self.sinv(self.point(x_real), "real", "fourier")

        def g_sets(w1, w2):
            g1 = np.asarray([b.to_real(b.fourier_filter(w1, 0, ks[i], ks[i + 1])) for i in range(nks)])
            g2 = np.asarray([b.to_real(b.fourier_filter(w2, 0, ks[i], ks[i + 1])) for i in range(nks)])
            return g1, g2

        local = b.sightline == "local" and self.lmax > 0
        legs = {}

        def gl_maps(w, B):
            if not local:
                return [b.to_real(b.fourier_filter(w, l, ks[B], ks[B + 1])) for l in range(2, self.lmax + 1, 2)]
            key = id(w)
            if key not in legs:
                legs[key] = (w, [b.apply_fourier_harmonics(b.to_real(w), l) for l in range(2, self.lmax + 1, 2)])
            return [b.to_real(b.fourier_filter(h, 0, ks[B], ks[B + 1])) for h in legs[key][1]]

        Nh = b.modk_grid.shape
        Q = np.zeros((self.N_bins,) + Nh, dtype=np.complex128)           # 643
        # Q[A^-1 a] (compute_Q 'Ainv', 521-640)
        w1, w2 = b.applyAinv_fourier(a1), b.applyAinv_fourier(a2)
        g1, g2 = g_sets(w1, w2)
        for B in range(nks):
            gl1, gl2 = (gl_maps(w1, B), gl_maps(w2, B)) if self.lmax > 0 else ([], [])
            for A in range(B + 1):
                i1 = np.where((ab[:, 0] == A) & (ab[:, 1] == B))[0]
                i2 = np.where((ab[:, 1] == A) & (ab[:, 2] == B))[0]
                i3 = np.where((ab[:, 2] == B) & (ab[:, 0] == A))[0]
                if len(i1) + len(i2) + len(i3) == 0:
                    continue
                ft = [b.to_fourier(b.prod_real_diff(g1[A], g1[B], g2[A], g2[B]))]
                for l in range(2, self.lmax + 1, 2):
                    ft.append(b.to_fourier(b.prod_real_diff(g1[A], gl1[l // 2 - 1], g2[A], gl2[l // 2 - 1])))
                for ii in i1:                                            # leg b3, L_l on it
                    C, l = ab[ii, 2], ab[ii, 3]
                    if local and l > 0:
                        Q[ii] += b.to_fourier(b.apply_real_harmonics(b.fourier_filter(ft[0], 0, ks[C], ks[C + 1]), l))
                    else:
                        Q[ii] += b.fourier_filter(ft[0], l, ks[C], ks[C + 1])
                for ii in i2:                                            # leg b1
                    C, l = ab[ii, 0], ab[ii, 3]
                    Q[ii] += b.fourier_filter(ft[l // 2], 0, ks[C], ks[C + 1])
                for ii in i3:                                            # leg b2
                    C, l = ab[ii, 1], ab[ii, 3]
                    Q[ii] += b.fourier_filter(ft[l // 2], 0, ks[C], ks[C + 1])
        for i in range(self.N_bins):                                     # 662-666
            Q[i] = apply_filter(Q[i], None if self.const_mask else b.to_real(Q[i]))
        # Q[S^-1 P a] rows (compute_Q 'Sinv')
        if self.const_mask:
            w1, w2 = apply_filter(a1), apply_filter(a2)
        else:
            w1, w2 = apply_filter(None, ar1), apply_filter(None, ar2)
        g1, g2 = g_sets(w1, w2)
        fish = np.zeros((self.N_bins, self.N_bins))
        for B in range(nks):
            gl1, gl2 = (gl_maps(w1, B), gl_maps(w2, B)) if self.lmax > 0 else ([], [])
            for A in range(B + 1):
                these = np.where((ab[:, 2] == B) & (ab[:, 0] == A))[0]
                if len(these) == 0:
                    continue
                for l in range(0, self.lmax + 1, 2):
                    if l == 0:
                        ft = b.to_fourier(b.prod_real_diff(g1[A], g1[B], g2[A], g2[B]))
                    else:
                        ft = b.to_fourier(b.prod_real_diff(g1[A], gl1[l // 2 - 1], g2[A], gl2[l // 2 - 1]))
                    for ii in these[ab[these, 3] == l]:
                        s = ab[ii, 1]
                        fish[ii] = b.integrate_row(ft, Q, ks[s], ks[s + 1])
        fish = 0.5 * fish * b.volume / b.gridsize.prod() ** 2 / np.outer(sym, sym)   # 674
        if return_Q:
            return fish, Q
        return fish
