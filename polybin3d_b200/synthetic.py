"""Seeded synthetic inputs with the shapes and statistics of the benchmark workloads.

No dataset is involved anywhere: every field and mask is generated here from a seed,
on the host, in FP64 numpy, so the CUDA path and the oracle see identical inputs.

* fiducial spectrum  P(k) = 1e4 (k/0.1)^-1.5 exp(-(k/0.3)^2)  (Mpc/h)^3,  P(0) = 0
* Gaussian random field: white noise from numpy's default_rng(seed), coloured in Fourier
  space by sqrt(P(|k|) N^3 / V) on the k-grid of the estimator (fftshift order on the
  first two axes, 0..N/2 on the last)
* lognormal: delta = exp(delta_G - sigma^2/2) - 1 with sigma^2 = var(delta_G), float32
* survey-like mask: 1 inside a spherical shell about the box centre, restricted to the
  x,y,z>0 octant, with seeded spherical holes set to 0, float32
"""
import numpy as np
import scipy.fft


def fiducial_pk(k):
    k = np.asarray(k, dtype=np.float64)
    out = np.zeros_like(k)
    nz = k > 0
    out[nz] = 1e4 * (k[nz] / 0.1) ** -1.5 * np.exp(-(k[nz] / 0.3) ** 2)
    return out


def modk_grid(gridsize, boxsize):
    """|k| on the half-complex grid, same construction as the estimator's k-grid."""
    N = np.asarray(gridsize, dtype=int)
    L = np.asarray(boxsize, dtype=np.float64)
    kF = 2.0 * np.pi / L
    ka = [np.fft.fftshift(np.arange(-N[i] // 2, N[i] // 2)) * kF[i] for i in range(2)]
    ka += [np.arange(0, N[2] // 2 + 1) * kF[2]]
    kg = np.meshgrid(*ka, indexing="ij")
    return np.sqrt(kg[0] ** 2 + kg[1] ** 2 + kg[2] ** 2)


def _as3(x, dtype):
    x = np.atleast_1d(np.asarray(x, dtype=dtype))
    return np.repeat(x, 3) if x.size == 1 else x


def grf(gridsize, boxsize, seed, pk=fiducial_pk):
    """FP64 Gaussian random field with power spectrum pk."""
    N = _as3(gridsize, int)
    L = _as3(boxsize, np.float64)
    w = np.random.default_rng(seed).standard_normal(tuple(N))
    amp = np.sqrt(pk(modk_grid(N, L)) * N.prod() / L.prod())
    return scipy.fft.irfftn(scipy.fft.rfftn(w) * amp, s=tuple(N))


def lognormal(gridsize, boxsize, seed, pk=fiducial_pk):
    """float32 lognormal field exp(dG - s2/2) - 1, s2 = var(dG) in FP64."""
    dG = grf(gridsize, boxsize, seed, pk)
    s2 = dG.var()
    return (np.exp(dG - s2 / 2.0) - 1.0).astype(np.float32)


def shell_mask(gridsize, boxsize, r_in, r_out, n_holes, hole_r=(5.0, 20.0), hole_box=700.0, seed=0):
    """float32 mask: 1 for r_in < r < r_out and x,y,z > 0, minus n_holes seeded spheres.

    Voxel coordinate x_i = ((i + N/2) mod N - N/2) L/N (the fftshift real-space grid with
    box centre 0).  Hole centres uniform in [0, hole_box)^3, radii uniform in hole_r."""
    N = _as3(gridsize, int)
    L = _as3(boxsize, np.float64)
    ax = [(((np.arange(N[i]) + N[i] // 2) % N[i]) - N[i] // 2) * L[i] / N[i] for i in range(3)]
    x, y, z = np.meshgrid(*ax, indexing="ij")
    r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    m = ((r > r_in) & (r < r_out) & (x > 0) & (y > 0) & (z > 0)).astype(np.float32)
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, hole_box, size=(n_holes, 3))
    radii = rng.uniform(hole_r[0], hole_r[1], size=n_holes)
    for c, rad in zip(centres, radii):
        # restrict the test to the hole's bounding box for speed
        sel = [np.nonzero(np.abs(ax[i] - c[i]) <= rad)[0] for i in range(3)]
        if any(len(s) == 0 for s in sel):
            continue
        sx, sy, sz = np.ix_(*sel)
        d2 = (x[sx, sy, sz] - c[0]) ** 2 + (y[sx, sy, sz] - c[1]) ** 2 + (z[sx, sy, sz] - c[2]) ** 2
        blk = m[sx, sy, sz]
        blk[d2 < rad ** 2] = 0.0
        m[sx, sy, sz] = blk
    return m


def pk_table(kmax, n=4000):
    """Tabulated fiducial spectrum [k, P(k)] for the estimator's `Pk=` argument."""
    k = np.linspace(0.0, kmax, n)
    return np.asarray([k, np.maximum(fiducial_pk(k), 0.0)])
