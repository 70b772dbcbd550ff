/*
 * polybin3d_b200 — C ABI of the B200-native binned-polyspectrum hot path.
 *
 * Every entry point takes raw device pointers, element counts, a `pb_grid_t` describing
 * the Fourier grid, and a CUDA stream (as void*).  Nothing here allocates device memory:
 * scratch comes from the caller, sized by the matching *_workspace_size query.  Calls
 * are stream-ordered and never synchronise the host, so they can be captured in CUDA
 * graphs.  Status: 0 = ok, negative = error; pb_last_error() gives the message of the
 * last failure on the calling host thread.
 *
 * Layouts (C-contiguous, one "map" per slab):
 *   real map      double|float [n0][n1][n2]
 *   half spectrum complex      [n0][n1][n2/2+1], interleaved (re, im), numpy rfftn order:
 *                 index i on axes 0,1 is frequency i for i < n/2 and i - n otherwise;
 *                 index l on axis 2 is frequency l (0..n2/2).
 * Mode geometry is recomputed on the device bit-exactly as the reference builds it in
 * numpy (PolyBin3D/base.py:86-92, 111-116): k_i = (double)idx * kF_i,
 * |k| = sqrt((kx*kx + ky*ky) + kz*kz), mu = kz/|k|, deg = 1 + (kz > 0).
 * A mode is in bin [lo, hi) iff lo <= |k| && |k| < hi  (PolyBin3D/cython/utils.pyx:63).
 */
#ifndef POLYBIN3D_B200_H
#define POLYBIN3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PB_API __attribute__((visibility("default")))
#else
#define PB_API
#endif

#define PB_ABI_VERSION 2

#define PB_OK 0
#define PB_ERR_INVALID (-1)     /* bad argument (shape, size, null pointer, range)      */
#define PB_ERR_CUDA (-2)        /* CUDA runtime error                                    */
#define PB_ERR_CUFFT (-3)       /* cuFFT error                                           */
#define PB_ERR_WORKSPACE (-4)   /* caller workspace too small                            */
#define PB_ERR_UNSUPPORTED (-5) /* configuration not built / device not sm_100           */
#define PB_ERR_TIMEOUT (-6)     /* a bounded device wait expired                        */

#define PB_F32 0
#define PB_F64 1
/* pb_shell_synth / pb_shell_synth_tiled only: FP32 maps (and FP32 w) from a complex FP64  */
/* source spectrum, which the first pass reads and filters in FP64 before rounding once   */
#define PB_F32_SRC_F64 2

typedef struct pb_grid {
    int32_t n[3];      /* real-space grid; n[2] even                                        */
    int32_t flags;     /* bit 0 (PB_GRID_LOS): los[] holds the line of sight of mu          */
    double kf[3];      /* fundamental frequencies 2 pi / L_i                                */
    double los[3];     /* unit line-of-sight vector, read when flags & PB_GRID_LOS:         */
                       /* mu = (k . los)/|k|, the local-sightline mu grid of                */
                       /* PolyBin3D/base.py:111-116; otherwise mu = k_z/|k| (global)        */
} pb_grid_t;
#define PB_GRID_LOS 1

/* Library identity and errors.  No reference counterpart (the reference raises Python
 * exceptions: e.g. PolyBin3D/base.py:54, pspec.py:591). */
PB_API int pb_abi_version(void);
PB_API const char *pb_last_error(void);

/* ---------------------------------------------------------------------------------- */
/* Launch shapes of the kernels that have more than one good shape, chosen per host      */
/* thread (the autotuner of polybin3d_b200/autotune.py times the candidates on first use  */
/* and sets the winner before each call).  Zero in a field means the built-in default.   */
/* Results do not depend on these settings beyond FP summation order.  No reference      */
/* counterpart (the reference has no launch configuration).                              */
/* ---------------------------------------------------------------------------------- */
typedef struct pb_tuning {
    int32_t tc_tile;     /* tensor-core contraction: voxels per tile, 32, 64 or 128 (0: 128, */
                         /* smaller when a shape does not fit; a tiled map set takes 128)    */
    int32_t tc_stages;   /* its staging ring depth in tiles, 2..6 (0: what ~64 KB holds)     */
    int32_t tc_chain;    /* voxels summed in TMEM between FP64 folds: 256 .. 2048 (0: 512);    */
                         /* changes the FP32 rounding, so the autotuner leaves it alone      */
    int32_t red_method;  /* k-bin reduction of many rows: 1 lane per row, 2 mode tiles (0: auto) */
    int32_t red_warps;   /* lane-per-row reduction: warps per block, 1..8 (0: as 48 KB fit)   */
    int32_t red_waves;   /* lane-per-row reduction: blocks per SM per 32-row group, 1..32 (0: 8) */
    int32_t tc_wait;     /* tensor-core contraction waits: 1 suspending try_wait, 2 polling   */
                         /* test_wait on the MMA / operand path (0: 1)                        */
    int32_t tc_dsets;    /* its TMEM accumulator sets, 1 or 2 (0: 2 when they fit); one set   */
                         /* leaves columns for more operand buffers                           */
} pb_tuning_t;
PB_API int pb_set_tuning(const pb_tuning_t *t); /* NULL restores the defaults               */
PB_API int pb_get_tuning(pb_tuning_t *t);

/* ---------------------------------------------------------------------------------- */
/* 3-D real FFTs.  Replace PolyBin3D/base.py:176-229 (`to_fourier`, `to_real`) and the   */
/* plan set-up of base.py:256-302 (`_fft_setup`).  Forward r2c is unnormalised; the c2r  */
/* is unnormalised too (the 1/N^3 of numpy's irfftn is folded into the kernels that      */
/* write its input).  The c2r overwrites its input.                                      */
/* ---------------------------------------------------------------------------------- */
typedef struct pb_fft_plan pb_fft_plan;
#define PB_FFT_R2C 0
#define PB_FFT_C2R 1
PB_API int pb_fft_plan_create(const pb_grid_t *g, int batch, int precision, int direction,
                       pb_fft_plan **plan, size_t *workspace_bytes);
PB_API int pb_fft_exec(pb_fft_plan *plan, const void *in, void *out, void *workspace, void *stream);
PB_API int pb_fft_plan_destroy(pb_fft_plan *plan);

/* ---------------------------------------------------------------------------------- */
/* Spectral filter: writes n_maps half spectra in one pass over the grid.               */
/*   out[m](k) = [acc ? out[m](k) : 0] + scale[m] * w(k)^wpow[m] * src[src_idx[m]](k)    */
/*               * Theta(lo[m] <= |k| < hi[m]) * L_{l1[m]}(mu) * L_{l2[m]}(mu)            */
/* src == NULL means a source of 1 + 0i (used for binning functions of a weight grid).   */
/* w (real, same precision as the spectra) may be NULL (= 1); wpow in {-1,0,1,2}, where  */
/* -1 divides (0 where w == 0).  l1, l2 in {0,...,4}.  src and w live on grid g; out may */
/* live on another grid out_n[3] (NULL = g): each output mode reads the source mode of   */
/* the same frequency (0 if the source grid lacks it), so band-limited maps can move     */
/* between the data grid and a coarser map grid.  dst_idx (host, may be NULL = identity) */
/* sends entry m to output dst_idx[m]; outputs may repeat, which requires accumulate.    */
/* Replaces MapUtils.fourier_filter / fourier_filter_ll / prod_fourier / prod_fourier_  */
/* filter / div_fourier (PolyBin3D/cython/utils.pyx:213-338) and jax_utils.py:97-100.    */
/* ---------------------------------------------------------------------------------- */
#define PB_FILTER_MAX_MAPS 128
PB_API int pb_spectral_filter(const pb_grid_t *g, const int32_t *out_n, int precision, const void *src,
                              int64_t src_stride, void *out, int n_maps, const int32_t *src_idx,
                              const int32_t *dst_idx, const double *lo, const double *hi,
                              const int32_t *l1, const int32_t *l2, const double *scale,
                              const int32_t *wpow, const void *w, int accumulate, void *stream);

/* ---------------------------------------------------------------------------------- */
/* Band-limited map synthesis: pb_spectral_filter onto the output grid out_n followed by */
/* the unnormalised C2R transform of every output spectrum, in one call:                 */
/*   out[m](x) = sum_k F_m(k) e^{+2 pi i k.x / M},  F_m as in pb_spectral_filter          */
/* Replaces fourier_filter + to_real per bin (utils.pyx:283-320, base.py:199-229; the    */
/* g-maps of bspec.py:936-956).  F_m vanishes outside |k| < hi_m, so only those planes,  */
/* columns and rows are transformed (pruned Stockham transforms in shared memory; two    */
/* real output lines share one complex transform along z).  out: real [n_maps][M0][M1][M2] */
/* in `precision`; src == NULL stands for a unit spectrum (the binning functions).       */
/* At most 64 maps per call.  PB_ERR_UNSUPPORTED (use the filter + FFT                  */
/* pair) when a band reaches a grid's Nyquist frequency, an upper edge is infinite, or an */
/* output length has a prime factor other than 2, 3, 5.  Workspace from                 */
/* pb_shell_synth_workspace_size (same grids, precision and upper edges).                */
/* ---------------------------------------------------------------------------------- */
PB_API int pb_shell_synth_workspace_size(const pb_grid_t *g, const int32_t *out_n, int precision, int n_maps,
                                         const double *hi, size_t *bytes);
PB_API int pb_shell_synth(const pb_grid_t *g, const int32_t *out_n, int precision, const void *src,
                          int64_t src_stride, int n_maps, const int32_t *src_idx, const double *lo,
                          const double *hi, const int32_t *l1, const int32_t *l2, const double *scale,
                          const int32_t *wpow, const void *w, void *out, void *workspace,
                          size_t workspace_bytes, void *stream);
/* The same maps written as a tiled map set (f32 only; the first n_factor maps are the    */
/* pair factors; see pb_tiled_maps_bytes for the layout and the size of `out`), ready for */
/* pb_triplet_contract_tiled.                                                            */
PB_API int pb_shell_synth_tiled(const pb_grid_t *g, const int32_t *out_n, int precision, const void *src,
                                int64_t src_stride, int n_maps, int n_factor, const int32_t *src_idx,
                                const double *lo, const double *hi, const int32_t *l1, const int32_t *l2,
                                const double *scale, const int32_t *wpow, const void *w, void *out,
                                void *workspace, size_t workspace_bytes, void *stream);

/* Binned-weight filter (the backward of the k-bin reduction):                           */
/*   out(k) = scale * src(k) * w(k)^wpow * sum_e coef[e][b(k)] L_{ells[e]}(mu),           */
/* b(k) the bin of |k| in `edges` (host, nk bins), 0 outside all bins; coef is a device  */
/* FP64 array [n_ell][nk] (so it can be an autograd cotangent); wpow in [-2, 2] (negative */
/* divides, 0 where w == 0).  The vector-Jacobian product of the power-spectrum         */
/* numerator, whose rows are the Q-maps of PolyBin3D/pspec.py:443-456.                    */
PB_API int pb_binned_filter(const pb_grid_t *g, int precision, const void *src, void *out,
                            const double *edges, int nk, const int32_t *ells, int n_ell,
                            const double *coef, const void *w, int wpow, double scale, void *stream);

/* ---------------------------------------------------------------------------------- */
/* k-bin x Legendre reductions over the half spectrum, FP64 accumulation.                */
/*   mode PB_RED_ABS2  : f_r = |a_r|^2                 (IntegrationUtils.integrate,       */
/*                                                      utils.pyx:80-104)                 */
/*   mode PB_RED_CROSS : f_r = Re(a * conj(b_r))       (cross_integrate, utils.pyx:51-75) */
/*                       a is one spectrum, b holds n_rows spectra                        */
/*   mode PB_RED_REAL2 : f = w^2, w = a real per mode  (real_integrate_double,           */
/*                       (a == NULL: w = 1, mode counts) utils.pyx:109-134)              */
/*   out[r][e][b] = scale * sum_{lo_b<=|k|<hi_b} deg * f_r * L_{ells[2e]}(mu) L_{ells[2e+1]}(mu)
/* with lo_b = edges[b], hi_b = edges[b+1] (strictly increasing, host array, nk <= 64),  */
/* n_ell <= 9 (pairs of Legendre orders, host array).  out is device FP64,              */
/* accumulate != 0 adds into it.  Deterministic (fixed-order two-pass reduction).       */
/* ---------------------------------------------------------------------------------- */
#define PB_RED_ABS2 0
#define PB_RED_CROSS 1
#define PB_RED_REAL2 2
#define PB_RED_MAX_BINS 64
#define PB_RED_MAX_ELLS 9
PB_API int pb_bin_reduce_workspace_size(const pb_grid_t *g, int n_rows, int nk, int n_ell, size_t *bytes);
PB_API int pb_bin_reduce(const pb_grid_t *g, int precision, int mode, const void *a, const void *b,
                  int n_rows, int64_t row_stride, const double *edges, int nk,
                  const int32_t *ells, int n_ell, double scale, double *out, int accumulate,
                  void *workspace, size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------------------- */
/* Triplet contraction over real maps (the bispectrum cubic sum):                        */
/*   out[t] = scale * sum_x A[i1_t](x) * B[i2_t](x) * C[i3_t](x)                          */
/* A, B, C: n_a / n_b / n_c maps of n_vox voxels each (may alias).  Replaces assemble_b3 */
/* and sum_triplet (PolyBin3D/cython/utils.pyx:614-636, 357-366; jax_utils.py:279-291).  */
/*                                                                                       */
/* pb_triplet_plan (host only) turns the host int32 list idx of n_trip (i1,i2,i3) rows   */
/* into a table (work items of the CUDA-core form, the pair rows and the triplet ->      */
/* (pair, i3) map of the tensor-core form) and its counts; call with table == NULL to    */
/* get its size, then copy the table to device memory once and pass it with the counts  */
/* to pb_triplet_contract.                                                              */
/* method PB_TRIPLET_SIMT: CUDA-core FMA form in the maps' precision, per-tile sums      */
/*   folded into FP64 registers.                                                         */
/* method PB_TRIPLET_TC: f32 maps; tcgen05 tensor cores (sm_100a).  The pair products    */
/*   A[i1]*B[i2] (MMA M, 128 pairs per M-tile, in tensor memory) and the C maps (MMA N)   */
/*   are split into bf16 hi + lo; per 16 voxels two MMAs accumulate the hi*hi, hi*lo and  */
/*   lo*hi terms in FP32 in TMEM, folded into FP64 every 512 voxels.  Any pair count (in  */
/*   launches of up to 512 pairs); at most 64 C maps and 256 maps per set (else           */
/*   PB_ERR_UNSUPPORTED).                                                                */
/* Output FP64 on the device, deterministic for a given device.                          */
/* ---------------------------------------------------------------------------------- */
#define PB_TRIPLET_SIMT 0
#define PB_TRIPLET_TC 1
/* counts[4]: n_items (CUDA-core work items), n_pairs (distinct (i1,i2)), n_groups, n_trip */
PB_API int pb_triplet_plan(int n_a, int n_b, int n_c, const int32_t *idx, int n_trip, void *table,
                           size_t *table_bytes, int32_t *counts);
PB_API int pb_triplet_workspace_size(int precision, int method, int64_t n_vox, const int32_t *counts,
                                     int n_c, size_t *bytes);
PB_API int pb_triplet_contract(int precision, int method, const void *A, int n_a, const void *B, int n_b,
                               const void *C, int n_c, int64_t n_vox, const void *table,
                               const int32_t *counts, double scale, double *out, void *workspace,
                               size_t workspace_bytes, void *stream);

/* Tiled map sets: the tensor-core contraction's staging layout in device memory, so that */
/* one contiguous copy stages a tile of 128 voxels.  n_maps f32 maps of n_vox voxels, of  */
/* which the first n_factor (1 <= n_factor <= n_maps) are pair factors.  Per tile t, at    */
/* byte t * 512 (F + P) (F = n_factor rounded up to 8, P = n_maps rounded up to 16):       */
/*  - factor slabs, 4 x F x 128 bytes: slab s (voxels 32s..32s+31 of the tile), row m     */
/*    (factor map m) holds the FP32 values, 16-byte chunk c (voxels 4c..4c+3) at chunk     */
/*    position c XOR (m mod 8);                                                           */
/*  - C operand, 8 x 2P x 32 bytes: step k (voxels 16k..16k+15 of the tile), row r holds   */
/*    the bf16 hi part rn(x) of map r (r < P) or the lo part rn(x - hi) of map r - P, the   */
/*    16-byte half h (voxels 8h..8h+7) at half position h XOR ((r / 4) mod 2) -- the        */
/*    32-byte-swizzled K-major layout of a tcgen05 MMA operand, one K step per 8-row atom. */
/* Voxels past n_vox hold zeros.  pb_tile_maps converts [n_maps][n_vox] maps;              */
/* pb_shell_synth_tiled writes the layout directly.  pb_triplet_contract_tiled is          */
/* pb_triplet_contract with A = B = C = the set (table and counts from pb_triplet_plan(    */
/* n_maps, n_maps, n_maps, ...) whose pair indices i1, i2 are below n_factor -- other      */
/* pairs make the call's outputs NaN -- and workspace from pb_triplet_workspace_size(      */
/* PB_F32, PB_TRIPLET_TC, n_vox, counts, n_maps)); method PB_TRIPLET_TC only, at most 64   */
/* maps.  No reference counterpart (the reference's maps are plain numpy arrays); the     */
/* contraction replaces the same assemble_b3 call.                                       */
PB_API int pb_tiled_maps_bytes(int n_maps, int n_factor, int64_t n_vox, size_t *bytes);
PB_API int pb_tile_maps(const void *maps, int n_maps, int n_factor, int64_t n_vox, void *tiled, void *stream);
PB_API int pb_triplet_contract_tiled(int method, const void *maps, int n_maps, int n_factor, int64_t n_vox,
                                     const void *table, const int32_t *counts, double scale, double *out,
                                     void *workspace, size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------------------- */
/* Bilinear maps (the adjoint of the triplet contraction with respect to its maps):       */
/*   out[o](x) = sum_t [o_t == o] c_t G[i_t](x) G[j_t](x)                                  */
/* The derivative of sum_t gamma_t sum_x G_a G_b G_c with respect to map G_o gathers, per */
/* output map, every leg ending on it: one map per leg instead of one product map per pair */
/* of maps, so the bispectrum gradient needs one forward transform per (bin, multipole)    */
/* leg instead of one per pair (the per-pair Q-map construction of PolyBin3D/bspec.py:     */
/* 600-640, as used for the autograd backward).                                           */
/* pb_bilinear_plan (host only) validates the host term lists (o < n_out, i, j < n_g),     */
/* merges duplicates and writes a table (call with table == NULL for its size and term    */
/* count n_table); copy it to 16-byte aligned device memory and pass it with n_table and   */
/* the same n_g and n_out to pb_bilinear_maps.  G: n_g real maps of n_vox voxels; out:     */
/* n_out maps, every one written (zeros where an output has no term).  At most 128 maps    */
/* and 4096 outputs.                                                                       */
/* ---------------------------------------------------------------------------------- */
PB_API int pb_bilinear_plan(int n_g, int n_out, const int32_t *o, const int32_t *i, const int32_t *j,
                            const double *c, int n_terms, void *table, size_t *table_bytes, int32_t *n_table);
PB_API int pb_bilinear_maps(int precision, int64_t n_vox, const void *G, int n_g, const void *table, int n_table,
                            int n_out, void *out, void *stream);

/* ---------------------------------------------------------------------------------- */
/* Real-space elementwise products.                                                      */
/*   PB_EW_MUL      : out = s * x * y                  (prod_real, utils.pyx:248-260)     */
/*   PB_EW_PRODDIFF : out = s * (x*y - z*u)            (prod_real_diff, utils.pyx:371-383)*/
/*   PB_EW_WIDEN    : out = (double) x, exact; x FP32 (precision PB_F32), out FP64; y, z, */
/*                    u, s unused (the FP32 data field before an FP64 r2c, base.py:176-198)*/
/* n elements; y is read at i % y_period when y_period > 0 (one mask over a batch of     */
/* maps; MUL only); z/u may be NULL where unused; out may alias x (not for WIDEN).       */
/* ---------------------------------------------------------------------------------- */
#define PB_EW_MUL 0
#define PB_EW_PRODDIFF 1
#define PB_EW_WIDEN 2
PB_API int pb_elementwise(int precision, int op, int64_t n, const void *x, const void *y, int64_t y_period,
                          const void *z, const void *u, double s, void *out, void *stream);

/* ---------------------------------------------------------------------------------- */
/* Gaussian random field from white noise (PolyBin3D/base.py:305-353):                   */
/*   r = noise_re + i noise_im on the full grid, r[0,0,0] = 0,                            */
/*   a(k) = 0.5 (r(k) + conj(r(-k))) on the half grid, times amp(k) * scale              */
/* noise: FP64 [n_batch][n0][n1][n2] each; amp: FP64 half grid (sqrt(P) * W); out: half  */
/* spectra [n_batch] in `precision`.                                                     */
/* ---------------------------------------------------------------------------------- */
PB_API int pb_grf_from_noise(const pb_grid_t *g, int precision, const double *noise_re,
                      const double *noise_im, int n_batch, const double *amp, double scale,
                      void *out, void *stream);

/* The same field with the white noise drawn on the device: for field b with seed       */
/* seeds[b] (device int64 array, so a captured graph can be replayed with new seeds) the */
/* noise at full-grid voxel p is a Box-Muller pair (re, im) of the first two words of    */
/* Philox4x32-10 (Salmon et al., SC'11) with key = seed and counter = (p, 0x5A17, 0).   */
/* Deterministic per (seed, voxel), independent of the batch it is drawn in; it is NOT   */
/* the reference's MT19937 stream (use pb_grf_from_noise for reference-identical noise). */
#define PB_PHILOX_DOMAIN 0x5A17u
PB_API int pb_grf_philox(const pb_grid_t *g, int precision, const int64_t *seeds, int n_batch,
                         const double *amp, double scale, void *out, void *stream);

/* ---------------------------------------------------------------------------------- */
/* Batched pair products of real maps:                                                   */
/*   out[p] = s * (X[i_p] * Y[j_p] - Z[i_p] * U[j_p])   (Z = U = NULL: s * X[i_p] Y[j_p]) */
/* pairs: host int32 (i_p, j_p) rows.  The g-map pair differences of the bispectrum      */
/* Fisher (prod_real_diff, utils.pyx:371-383, called at PolyBin3D/bspec.py:591-613).     */
/* ---------------------------------------------------------------------------------- */
#define PB_PAIR_MAX 256
PB_API int pb_pair_products(int precision, int64_t n_vox, const void *X, const void *Y, const void *Z,
                            const void *U, const int32_t *pairs, int n_pairs, double s, void *out,
                            void *stream);

/* ---------------------------------------------------------------------------------- */
/* Fisher rows over one k-shell (IntegrationUtils.integrate_row, utils.pyx:162-179,      */
/* called per row at PolyBin3D/bspec.py:597):                                            */
/*   out[out_row[r] * out_stride + j] = scale * sum_{i < n_modes} deg(m_i)               */
/*                                      * Re(conj(F[row_key[r]](m_i)) * Q[j](m_i))        */
/* for r < n_rows (<= 32), j < n_cols.  modes: device int64 list of the shell's half-    */
/* grid indices (the modes with lo <= |k| < hi); F: n_f half spectra; Q: n_cols half     */
/* spectra; row_key/out_row: host int32.  Deterministic chunked FP64 sums.               */
/* ---------------------------------------------------------------------------------- */
PB_API int pb_shell_rows_workspace_size(int64_t n_modes, int n_rows, int n_cols, size_t *bytes);
PB_API int pb_shell_rows(const pb_grid_t *g, int precision, const void *F, int n_f, const void *Q,
                         int n_cols, const int64_t *modes, int64_t n_modes, const int32_t *row_key,
                         const int32_t *out_row, int n_rows, double scale, double *out,
                         int64_t out_stride, void *workspace, size_t workspace_bytes, void *stream);

/* ---------------------------------------------------------------------------------- */
/* pb_bin_reduce_noalloc: pb_bin_reduce for callers that cannot allocate device memory   */
/* (a binding that only forwards the pointers it was given, or a process whose GPU       */
/* memory belongs to another framework's pool).  No counterpart in the reference.        */
/* Same arguments and results as pb_bin_reduce minus the workspace: the partial sums go  */
/* to a fixed 2 MiB device array inside the library (PB_BIN_REDUCE_NOALLOC_MAX_DOUBLES   */
/* doubles, held on every GPU that loads the library until exit).  Fails with           */
/* PB_ERR_INVALID when n_rows * nk * n_ell exceeds it.  The first call on a device looks */
/* up the array's device address and should come before any stream capture; the address */
/* is kept for the process's life (no calls after a cudaDeviceReset).  All calls share   */
/* the array: calls that overlap on the GPU race and must be serialised.                 */
/* ---------------------------------------------------------------------------------- */
#define PB_BIN_REDUCE_NOALLOC_MAX_DOUBLES 262144
PB_API int pb_bin_reduce_noalloc(const pb_grid_t *g, int precision, int mode, const void *a,
                                 const void *b, int n_rows, int64_t row_stride, const double *edges,
                                 int nk, const int32_t *ells, int n_ell, double scale, double *out,
                                 int accumulate, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* POLYBIN3D_B200_H */
