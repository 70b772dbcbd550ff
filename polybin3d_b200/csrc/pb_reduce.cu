// k-bin x Legendre reductions over half spectra (the power-spectrum binning pass) and
// the per-shell Fisher-row contraction.  FP64 accumulation, deterministic two-pass sums.
#include <algorithm>
#include <string>
#include <vector>
#include "pb_common.cuh"

namespace pb {

struct RedParams {
    double edges[PB_RED_MAX_BINS + 1];
    int8_t la[PB_RED_MAX_ELLS];
    int8_t lb[PB_RED_MAX_ELLS];
    int32_t nk;
    int32_t n_ell;
};

constexpr int RED_THREADS = 256;
constexpr int RED_CHUNK = 4;  // consecutive modes per thread per step (same kz line, mostly same bin)

static int red_blocks(const Grid &G) {
    int64_t per_block = (int64_t)RED_THREADS * RED_CHUNK;
    int64_t b = (G.nhalf + per_block - 1) / per_block;
    int64_t cap = (int64_t)num_sms() * 2;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, cap));
}

// bin b with edges[b] <= k < edges[b+1], or -1
__device__ __forceinline__ int find_bin(const double *edges, int nk, double k) {
    if (!(edges[0] <= k) || !(k < edges[nk])) return -1;
    int lo = 0, hi = nk;  // invariant: edges[lo] <= k < edges[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (edges[mid] <= k) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <typename T, int MODE>
__global__ void __launch_bounds__(RED_THREADS) binred_kernel(Grid g, const typename cplx<T>::type *a,
                                                            const typename cplx<T>::type *b, const T *w,
                                                            int64_t row_stride, RedParams p, double *partials) {
    using C = typename cplx<T>::type;
    __shared__ double acc[PB_RED_MAX_ELLS * PB_RED_MAX_BINS];
    __shared__ double edges[PB_RED_MAX_BINS + 1];
    const int nk = p.nk, ne = p.n_ell;
    for (int i = threadIdx.x; i < ne * nk; i += blockDim.x) acc[i] = 0.0;
    for (int i = threadIdx.x; i <= nk; i += blockDim.x) edges[i] = p.edges[i];
    __syncthreads();
    const int row = blockIdx.y;
    const C *arow = (MODE == PB_RED_ABS2) ? a + (int64_t)row * row_stride : a;
    const C *brow = (MODE == PB_RED_CROSS) ? b + (int64_t)row * row_stride : nullptr;
    const int64_t step = (int64_t)gridDim.x * blockDim.x * RED_CHUNK;
    for (int64_t base = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * RED_CHUNK; base < g.nhalf;
         base += step) {
        int cur = -1;
        double run[PB_RED_MAX_ELLS];
#pragma unroll
        for (int e = 0; e < PB_RED_MAX_ELLS; ++e) run[e] = 0.0;
        const int64_t end = min(base + RED_CHUNK, g.nhalf);
        for (int64_t idx = base; idx < end; ++idx) {
            Mode md = mode_of(g, idx);
            int bin = find_bin(edges, nk, md.k);
            if (bin != cur) {
                if (cur >= 0) {
#pragma unroll
                    for (int e = 0; e < PB_RED_MAX_ELLS; ++e)
                        if (e < ne) atomicAdd(&acc[e * nk + cur], run[e]);
                }
#pragma unroll
                for (int e = 0; e < PB_RED_MAX_ELLS; ++e) run[e] = 0.0;
                cur = bin;
            }
            if (bin < 0) continue;
            double f;
            if (MODE == PB_RED_ABS2) {
                C v = arow[idx];
                f = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
            } else if (MODE == PB_RED_CROSS) {
                C u = arow[idx], v = brow[idx];
                f = (double)u.x * (double)v.x + (double)u.y * (double)v.y;
            } else {
                double v = w ? (double)w[idx] : 1.0;
                f = v * v;
            }
            f *= md.deg;
#pragma unroll
            for (int e = 0; e < PB_RED_MAX_ELLS; ++e)
                if (e < ne) run[e] += f * legendre(p.la[e], md.mu) * legendre(p.lb[e], md.mu);
        }
        if (cur >= 0) {
#pragma unroll
            for (int e = 0; e < PB_RED_MAX_ELLS; ++e)
                if (e < ne) atomicAdd(&acc[e * nk + cur], run[e]);
        }
    }
    __syncthreads();
    double *dst = partials + ((int64_t)row * gridDim.x + blockIdx.x) * (ne * nk);
    for (int i = threadIdx.x; i < ne * nk; i += blockDim.x) dst[i] = acc[i];
}

// Many rows over the same modes (the Fisher rows: CROSS of one spectrum with N_bins Q rows,
// or ABS2 of a batch).  The mode geometry -- bin, degeneracy x Legendre weights, the shared
// spectrum a -- is computed once per tile of modes into shared memory and then used by every
// row of the group, instead of once per row: the FP64 |k|, mu, bin search and Legendre
// polynomials no longer scale with the row count, and each row is one streaming read.
constexpr int RR_TILE = 512;                 // modes per tile (2 per thread)
constexpr int RR_PER = RR_TILE / RED_THREADS;
constexpr int RR_ACC_DOUBLES = 6144;         // shared accumulators per block (48 KB)
constexpr int RR_RB = 8;                     // rows loaded ahead per thread

// accumulator doubles rounded up to an even count, so the double2 tile after them is aligned
__host__ __device__ __forceinline__ size_t rr_acc_len(int rows, int ne, int nk) {
    return ((size_t)rows * ne * nk + 1) & ~(size_t)1;
}

template <typename T, int MODE>
__global__ void __launch_bounds__(RED_THREADS) binred_rows_kernel(Grid g, const typename cplx<T>::type *a,
                                                                 const typename cplx<T>::type *b,
                                                                 int64_t row_stride, RedParams p, int n_rows,
                                                                 int rows_per_group, double *partials) {
    using C = typename cplx<T>::type;
    extern __shared__ __align__(16) unsigned char rr_smem[];
    const int nk = p.nk, ne = p.n_ell;
    const int r0 = blockIdx.y * rows_per_group;
    const int nr = min(rows_per_group, n_rows - r0);
    double *acc = reinterpret_cast<double *>(rr_smem);          // [nr][ne][nk]
    double *wt = acc + rr_acc_len(rows_per_group, ne, nk);       // [ne][RR_TILE]
    double2 *as = reinterpret_cast<double2 *>(wt + (size_t)ne * RR_TILE);  // [RR_TILE] (CROSS)
    int *bins = reinterpret_cast<int *>(as + RR_TILE);            // [RR_TILE]
    __shared__ double edges[PB_RED_MAX_BINS + 1];
    for (int i = threadIdx.x; i < nr * ne * nk; i += blockDim.x) acc[i] = 0.0;
    for (int i = threadIdx.x; i <= nk; i += blockDim.x) edges[i] = p.edges[i];
    const int64_t n_tiles = (g.nhalf + RR_TILE - 1) / RR_TILE;
    for (int64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int64_t t0 = tile * RR_TILE;
        __syncthreads();  // previous tile's readers are done (and the set-up above is visible)
        for (int j = threadIdx.x; j < RR_TILE; j += blockDim.x) {
            const int64_t idx = t0 + j;
            int bin = -1;
            if (idx < g.nhalf) {
                const Mode md = mode_of(g, idx);
                bin = find_bin(edges, nk, md.k);
                if (bin >= 0) {
#pragma unroll
                    for (int e = 0; e < PB_RED_MAX_ELLS; ++e)
                        if (e < ne) wt[e * RR_TILE + j] = md.deg * legendre(p.la[e], md.mu) * legendre(p.lb[e], md.mu);
                }
                if (MODE == PB_RED_CROSS) {
                    const C v = a[idx];
                    as[j] = make_double2((double)v.x, (double)v.y);
                }
            }
            bins[j] = bin;
        }
        __syncthreads();
        // lane <-> consecutive mode (coalesced row reads).  Consecutive modes mostly share a
        // bin, so a warp first sums each contiguous run of equal bins with a segmented
        // shuffle reduction and only the run's first lane adds to shared memory: one atomic
        // per run and Legendre order instead of one per mode on the same address.
        const int lane = threadIdx.x & 31;
        for (int pass = 0; pass < RR_PER; ++pass) {
            const int j = pass * RED_THREADS + threadIdx.x;
            const int bin = bins[j];
            const bool head = lane == 0 || bins[j - 1] != bin;
            const unsigned heads = __ballot_sync(0xffffffffu, head);
            const int seg = __popc(heads & (0xffffffffu >> (31 - lane)));  // run index of this lane
            unsigned same = 0;                                              // bit k: lane + 2^k in my run
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                const int o = 1 << k;
                const int sg = __shfl_down_sync(0xffffffffu, seg, o);
                if (lane + o < 32 && sg == seg) same |= 1u << k;
            }
            double2 u = make_double2(0.0, 0.0);
            if (MODE == PB_RED_CROSS && bin >= 0) u = as[j];
            double w[PB_RED_MAX_ELLS];
#pragma unroll
            for (int e = 0; e < PB_RED_MAX_ELLS; ++e) w[e] = (e < ne && bin >= 0) ? wt[e * RR_TILE + j] : 0.0;
            // RR_RB rows' values are loaded before any of them is reduced, so each thread
            // keeps RR_RB independent reads in flight
            const C *src = (MODE == PB_RED_CROSS) ? b : a;
            for (int rb = 0; rb < nr; rb += RR_RB) {
                C vals[RR_RB];
#pragma unroll
                for (int q = 0; q < RR_RB; ++q) {
                    vals[q].x = 0;
                    vals[q].y = 0;
                    if (bin >= 0 && rb + q < nr) vals[q] = src[(int64_t)(r0 + rb + q) * row_stride + t0 + j];
                }
#pragma unroll
                for (int q = 0; q < RR_RB; ++q) {
                    if (rb + q >= nr) break;
                    double f;
                    if (MODE == PB_RED_CROSS) f = u.x * (double)vals[q].x + u.y * (double)vals[q].y;
                    else f = (double)vals[q].x * (double)vals[q].x + (double)vals[q].y * (double)vals[q].y;
                    double *accr = acc + (size_t)(rb + q) * ne * nk;
#pragma unroll
                    for (int e = 0; e < PB_RED_MAX_ELLS; ++e) {
                        if (e >= ne) break;
                        double v = f * w[e];
#pragma unroll
                        for (int k = 0; k < 5; ++k) {
                            const double up = __shfl_down_sync(0xffffffffu, v, 1 << k);
                            if (same & (1u << k)) v += up;
                        }
                        if (head && bin >= 0) atomicAdd(&accr[e * nk + bin], v);
                    }
                }
            }
        }
    }
    __syncthreads();
    for (int r = 0; r < nr; ++r) {
        double *dst = partials + ((int64_t)(r0 + r) * gridDim.x + blockIdx.x) * (ne * nk);
        for (int i = threadIdx.x; i < ne * nk; i += blockDim.x) dst[i] = acc[(size_t)r * ne * nk + i];
    }
}

// ------------------------------------------------------------------------------------
// Many rows, one lane per row.  The mode geometry (bin and deg x L_la L_lb per mode, FP64)
// is tabulated once per call by binred_geom_kernel.  A warp then walks kz lines of the half
// grid; each lane reads ITS row's values along the line (8 consecutive modes = one 128-byte
// segment for complex128) while the geometry and the shared spectrum are warp-uniform
// broadcasts.  All lanes see the same mode sequence, so a bin change is a uniform branch:
// the sums of the current bin stay in registers and are added to the lane's slot of the
// warp's shared-memory accumulators [bin][e][lane] only when the bin changes (no shuffles,
// no atomics, fixed order: deterministic).  Only the part of each line inside the binned
// range is read (|k| grows along a kz line, so it is one contiguous run of modes).
// ------------------------------------------------------------------------------------
constexpr int BL_MODES = 4;  // modes per lane per step (the next step's values load meanwhile)

__global__ void binred_geom_kernel(Grid g, RedParams p, int8_t *mbin, double *mw) {
    __shared__ double edges[PB_RED_MAX_BINS + 1];
    for (int i = threadIdx.x; i <= p.nk; i += blockDim.x) edges[i] = p.edges[i];
    __syncthreads();
    const int ne = p.n_ell;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < g.nhalf;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const Mode md = mode_of(g, idx);
        const int bin = find_bin(edges, p.nk, md.k);
        mbin[idx] = (int8_t)bin;
        if (bin >= 0) {
#pragma unroll
            for (int e = 0; e < PB_RED_MAX_ELLS; ++e)
                if (e < ne) mw[idx * ne + e] = md.deg * legendre(p.la[e], md.mu) * legendre(p.lb[e], md.mu);
        }
    }
}

template <typename T, int MODE, int NE>
__global__ void __launch_bounds__(256) binred_lanes_kernel(Grid g, const typename cplx<T>::type *a,
                                                           const typename cplx<T>::type *b, int64_t row_stride,
                                                           int n_rows, int nk, const int8_t *mbin, const double *mw,
                                                           double *partials) {
    using C = typename cplx<T>::type;
    constexpr int S = BL_MODES;
    extern __shared__ __align__(16) double bl_acc[];  // [warp][bin][e][32]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int per = nk * NE;
    double *wacc = bl_acc + (size_t)warp * per * 32;
    for (int i = threadIdx.x; i < nw * per * 32; i += blockDim.x) bl_acc[i] = 0.0;
    __syncthreads();
    const int row = blockIdx.y * 32 + lane;
    const bool live = row < n_rows;
    const C *brow = b + (int64_t)(live ? row : 0) * row_stride;
    const int64_t n_lines = (int64_t)g.n0 * g.n1;
    const int nh2 = g.nh2;
    double r[NE];
#pragma unroll
    for (int e = 0; e < NE; ++e) r[e] = 0.0;
    int cur = -1;
    for (int64_t line = (int64_t)blockIdx.x * nw + warp; line < n_lines; line += (int64_t)gridDim.x * nw) {
        const int64_t base = line * nh2;
        // the binned run [l_lo, l_hi) of this line
        int l_lo = nh2, l_hi = 0;
        for (int l0 = 0; l0 < nh2; l0 += 32) {
            const int l = l0 + lane;
            const bool in = l < nh2 && mbin[base + l] >= 0;
            const unsigned m = __ballot_sync(0xffffffffu, in);
            if (m) {
                l_lo = min(l_lo, l0 + __ffs(m) - 1);
                l_hi = l0 + 32 - __clz(m);
            }
        }
        if (l_lo >= l_hi) continue;
        // software pipeline: the row values of step s + 1 are in flight while step s is summed
        C v[S];
#pragma unroll
        for (int k = 0; k < S; ++k) {
            v[k].x = 0;
            v[k].y = 0;
            if (live && l_lo + k < l_hi) v[k] = brow[base + l_lo + k];
        }
        for (int l0 = l_lo; l0 < l_hi; l0 += S) {
            C nv[S];
#pragma unroll
            for (int k = 0; k < S; ++k) {
                nv[k].x = 0;
                nv[k].y = 0;
                if (live && l0 + S + k < l_hi) nv[k] = brow[base + l0 + S + k];
            }
            // this step's geometry and shared spectrum, loaded before any of it is used
            int bn[S];
            C av[S];
            double w[S][NE];
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const int64_t idx = base + l0 + k;
                const bool in = l0 + k < l_hi;
                bn[k] = in ? (int)mbin[idx] : -2;
                if (MODE == PB_RED_CROSS) {
                    av[k].x = 0;
                    av[k].y = 0;
                    if (in) av[k] = a[idx];
                }
#pragma unroll
                for (int e = 0; e < NE; ++e) w[k][e] = in ? mw[idx * NE + e] : 0.0;
            }
#pragma unroll
            for (int k = 0; k < S; ++k) {
                if (bn[k] == -2) break;
                if (bn[k] != cur) {
#pragma unroll
                    for (int e = 0; e < NE; ++e) {
                        if (cur >= 0) wacc[(cur * NE + e) * 32 + lane] += r[e];
                        r[e] = 0.0;
                    }
                    cur = bn[k];
                }
                if (bn[k] < 0) continue;
                double f;
                if (MODE == PB_RED_CROSS)
                    f = (double)av[k].x * (double)v[k].x + (double)av[k].y * (double)v[k].y;
                else
                    f = (double)v[k].x * (double)v[k].x + (double)v[k].y * (double)v[k].y;
#pragma unroll
                for (int e = 0; e < NE; ++e) r[e] += f * w[k][e];
            }
#pragma unroll
            for (int k = 0; k < S; ++k) v[k] = nv[k];
        }
    }
#pragma unroll
    for (int e = 0; e < NE; ++e)
        if (cur >= 0) wacc[(cur * NE + e) * 32 + lane] += r[e];
    __syncthreads();
    // warps' sums in fixed order -> this block's partial of each row
    for (int i = threadIdx.x; i < per * 32; i += blockDim.x) {
        const int ln = i & 31, be = i >> 5;  // be = bin * NE + e
        const int rr = blockIdx.y * 32 + ln;
        if (rr >= n_rows) continue;
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += bl_acc[((size_t)w * per + be) * 32 + ln];
        const int bin = be / NE, e = be - bin * NE;
        partials[((int64_t)rr * gridDim.x + blockIdx.x) * per + e * nk + bin] = s;
    }
}

struct LanesLaunch {
    int nw, gx;
    size_t smem;
    size_t geom_bytes;   // mbin (nhalf bytes, padded to 256) + mw (nhalf * n_ell doubles)
};

// the lane-per-row kernel serves many rows with small (bins x multipoles) accumulators
static bool lanes_plan(const Grid &G, int n_rows, int nk, int n_ell, LanesLaunch *L) {
    const pb_tuning_t &tu = tuning();
    if (tu.red_method == 2) return false;
    if (n_rows < (tu.red_method == 1 ? 1 : 16)) return false;
    const size_t per_warp = (size_t)nk * n_ell * 32 * sizeof(double);
    if (per_warp > 48 * 1024) return false;
    const size_t fit = std::max<size_t>(1, (48 * 1024) / per_warp);
    L->nw = tu.red_warps > 0 ? (int)std::min<size_t>((size_t)tu.red_warps, 2 * fit) : (int)std::min<size_t>(4, fit);
    L->smem = per_warp * L->nw;
    if (L->smem > 96 * 1024) return false;
    const int64_t n_lines = (int64_t)G.n0 * G.n1;
    const int groups = (n_rows + 31) / 32;
    const int waves = tu.red_waves > 0 ? tu.red_waves : 8;
    int64_t gx = ((int64_t)waves * num_sms() + groups - 1) / groups;
    gx = std::min<int64_t>(gx, (n_lines + L->nw - 1) / L->nw);
    L->gx = (int)std::max<int64_t>(1, gx);
    L->geom_bytes = ((size_t)G.nhalf + 255) / 256 * 256 + (size_t)G.nhalf * n_ell * sizeof(double);
    return true;
}

__global__ void binred_finalize(const double *partials, int n_blocks, int per_row, int n_rows, double scale,
                                double *out, int accumulate) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_rows * per_row) return;
    int row = t / per_row, j = t - row * per_row;
    const double *src = partials + (int64_t)row * n_blocks * per_row + j;
    double s = 0.0;
    for (int blk = 0; blk < n_blocks; ++blk) s += src[(int64_t)blk * per_row];
    s *= scale;
    out[t] = accumulate ? out[t] + s : s;
}

}  // namespace pb

using namespace pb;

extern "C" int pb_bin_reduce_workspace_size(const pb_grid_t *g, int n_rows, int nk, int n_ell, size_t *bytes) {
    Grid G;
    int st = make_grid(g, &G);
    if (st) return st;
    if (!bytes) return fail(PB_ERR_INVALID, "bytes is NULL");
    if (n_rows < 1 || nk < 1 || n_ell < 1) return fail(PB_ERR_INVALID, "pb_bin_reduce: empty reduction");
    *bytes = (size_t)n_rows * red_blocks(G) * nk * n_ell * sizeof(double);
    LanesLaunch L;
    if (lanes_plan(G, n_rows, nk, n_ell, &L))
        *bytes = std::max(*bytes, L.geom_bytes + (size_t)n_rows * L.gx * nk * n_ell * sizeof(double));
    return PB_OK;
}

extern "C" int pb_bin_reduce(const pb_grid_t *g, int precision, int mode, const void *a, const void *b,
                             int n_rows, int64_t row_stride, const double *edges, int nk, const int32_t *ells,
                             int n_ell, double scale, double *out, int accumulate, void *workspace,
                             size_t workspace_bytes, void *stream) {
    Grid G;
    int st = make_grid(g, &G);
    if (st) return st;
    if (nk < 1 || nk > PB_RED_MAX_BINS) return fail(PB_ERR_INVALID, "pb_bin_reduce: nk must be in [1, 64]");
    if (n_ell < 1 || n_ell > PB_RED_MAX_ELLS) return fail(PB_ERR_INVALID, "pb_bin_reduce: n_ell must be in [1, 9]");
    if (n_rows < 1 || n_rows > 65535) return fail(PB_ERR_INVALID, "pb_bin_reduce: n_rows must be in [1, 65535]");
    if (!edges || !ells || !out) return fail(PB_ERR_INVALID, "pb_bin_reduce: NULL argument");
    if (mode == PB_RED_ABS2 && !a) return fail(PB_ERR_INVALID, "pb_bin_reduce: ABS2 needs a");
    if (mode == PB_RED_CROSS && (!a || !b)) return fail(PB_ERR_INVALID, "pb_bin_reduce: CROSS needs a and b");
    if (mode < 0 || mode > 2) return fail(PB_ERR_INVALID, "pb_bin_reduce: bad mode");
    if (row_stride == 0) row_stride = G.nhalf;
    RedParams p;
    for (int i = 0; i <= nk; ++i) {
        p.edges[i] = edges[i];
        if (i > 0 && !(edges[i] > edges[i - 1]))
            return fail(PB_ERR_INVALID, "pb_bin_reduce: bin edges must be strictly increasing");
    }
    for (int e = 0; e < n_ell; ++e) {
        if (ells[2 * e] < 0 || ells[2 * e] > 4 || ells[2 * e + 1] < 0 || ells[2 * e + 1] > 4)
            return fail(PB_ERR_INVALID, "pb_bin_reduce: Legendre order must be in [0, 4]");
        p.la[e] = (int8_t)ells[2 * e];
        p.lb[e] = (int8_t)ells[2 * e + 1];
    }
    p.nk = nk;
    p.n_ell = n_ell;
    if (precision != PB_F32 && precision != PB_F64) return fail(PB_ERR_INVALID, "bad precision");
    int nb = red_blocks(G);
    size_t need = (size_t)n_rows * nb * nk * n_ell * sizeof(double);
    cudaStream_t s = as_stream(stream);
    LanesLaunch LL;
    if (mode != PB_RED_REAL2 && lanes_plan(G, n_rows, nk, n_ell, &LL)) {
        // geometry table, then one lane per row (binred_lanes_kernel)
        need = LL.geom_bytes + (size_t)n_rows * LL.gx * nk * n_ell * sizeof(double);
        if (!workspace || workspace_bytes < need)
            return fail(PB_ERR_WORKSPACE, "pb_bin_reduce: workspace too small (need " + std::to_string(need) + " bytes)");
        int8_t *mbin = (int8_t *)workspace;
        double *mw = (double *)((char *)workspace + ((size_t)G.nhalf + 255) / 256 * 256);
        double *partials = (double *)((char *)workspace + LL.geom_bytes);
        const int gg = (int)std::min<int64_t>((G.nhalf + 255) / 256, (int64_t)num_sms() * 8);
        binred_geom_kernel<<<gg, 256, 0, s>>>(G, p, mbin, mw);
        PB_LAUNCH_CHECK("pb_bin_reduce(geometry)");
        dim3 lgrid(LL.gx, (n_rows + 31) / 32);
        const void *rows = (mode == PB_RED_CROSS) ? b : a;
#define PB_BL_LAUNCH(T, M, NE)                                                                                  \
    do {                                                                                                        \
        PB_CUDA(cudaFuncSetAttribute(binred_lanes_kernel<T, M, NE>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                     (int)LL.smem));                                                            \
        binred_lanes_kernel<T, M, NE><<<lgrid, 32 * LL.nw, LL.smem, s>>>(G, (const cplx<T>::type *)a,          \
                                                                        (const cplx<T>::type *)rows, row_stride, \
                                                                        n_rows, nk, mbin, mw, partials);         \
    } while (0)
#define PB_BL_NE(T, M)                                        \
    switch (n_ell) {                                          \
        case 1: PB_BL_LAUNCH(T, M, 1); break;                 \
        case 2: PB_BL_LAUNCH(T, M, 2); break;                 \
        case 3: PB_BL_LAUNCH(T, M, 3); break;                 \
        case 4: PB_BL_LAUNCH(T, M, 4); break;                 \
        case 5: PB_BL_LAUNCH(T, M, 5); break;                 \
        case 6: PB_BL_LAUNCH(T, M, 6); break;                 \
        case 7: PB_BL_LAUNCH(T, M, 7); break;                 \
        case 8: PB_BL_LAUNCH(T, M, 8); break;                 \
        default: PB_BL_LAUNCH(T, M, 9); break;                \
    }
        if (precision == PB_F32) {
            if (mode == PB_RED_ABS2) PB_BL_NE(float, PB_RED_ABS2)
            else PB_BL_NE(float, PB_RED_CROSS)
        } else {
            if (mode == PB_RED_ABS2) PB_BL_NE(double, PB_RED_ABS2)
            else PB_BL_NE(double, PB_RED_CROSS)
        }
#undef PB_BL_NE
#undef PB_BL_LAUNCH
        PB_LAUNCH_CHECK("pb_bin_reduce(lanes)");
        const int per = nk * n_ell;
        const int total = per * n_rows;
        binred_finalize<<<(total + 255) / 256, 256, 0, s>>>(partials, LL.gx, per, n_rows, scale, out, accumulate);
        PB_LAUNCH_CHECK("pb_bin_reduce(finalize)");
        return PB_OK;
    }
    if (!workspace || workspace_bytes < need)
        return fail(PB_ERR_WORKSPACE, "pb_bin_reduce: workspace too small (need " + std::to_string(need) + " bytes)");
    double *partials = (double *)workspace;
    if (mode != PB_RED_REAL2) {
        // spectra: mode geometry once per tile for a group of rows (binred_rows_kernel)
        const int per = nk * n_ell;
        const int rpg = std::max(1, std::min(n_rows, RR_ACC_DOUBLES / per));
        const size_t smem = rr_acc_len(rpg, n_ell, nk) * sizeof(double) + (size_t)n_ell * RR_TILE * sizeof(double) +
                            (size_t)RR_TILE * (sizeof(double2) + sizeof(int));
        dim3 rgrid(nb, (n_rows + rpg - 1) / rpg);
#define PB_RR_LAUNCH(T, M)                                                                                   \
    do {                                                                                                     \
        PB_CUDA(cudaFuncSetAttribute(binred_rows_kernel<T, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                     (int)smem));                                                            \
        binred_rows_kernel<T, M><<<rgrid, RED_THREADS, smem, s>>>(G, (const cplx<T>::type *)a,              \
                                                                  (const cplx<T>::type *)b, row_stride, p,   \
                                                                  n_rows, rpg, partials);                    \
    } while (0)
        if (precision == PB_F32) {
            if (mode == PB_RED_ABS2) PB_RR_LAUNCH(float, PB_RED_ABS2);
            else PB_RR_LAUNCH(float, PB_RED_CROSS);
        } else if (precision == PB_F64) {
            if (mode == PB_RED_ABS2) PB_RR_LAUNCH(double, PB_RED_ABS2);
            else PB_RR_LAUNCH(double, PB_RED_CROSS);
        } else {
            return fail(PB_ERR_INVALID, "bad precision");
        }
#undef PB_RR_LAUNCH
        PB_LAUNCH_CHECK("pb_bin_reduce(rows)");
        const int total = per * n_rows;
        binred_finalize<<<(total + 255) / 256, 256, 0, s>>>(partials, nb, per, n_rows, scale, out, accumulate);
        PB_LAUNCH_CHECK("pb_bin_reduce(finalize)");
        return PB_OK;
    }
    dim3 grid(nb, n_rows);
#define PB_RED_LAUNCH(T, M)                                                                        \
    binred_kernel<T, M><<<grid, RED_THREADS, 0, s>>>(G, (const cplx<T>::type *)a, (const cplx<T>::type *)b, \
                                                      (const T *)a, row_stride, p, partials)
    if (precision == PB_F32) {
        if (mode == PB_RED_ABS2) PB_RED_LAUNCH(float, PB_RED_ABS2);
        else if (mode == PB_RED_CROSS) PB_RED_LAUNCH(float, PB_RED_CROSS);
        else PB_RED_LAUNCH(float, PB_RED_REAL2);
    } else if (precision == PB_F64) {
        if (mode == PB_RED_ABS2) PB_RED_LAUNCH(double, PB_RED_ABS2);
        else if (mode == PB_RED_CROSS) PB_RED_LAUNCH(double, PB_RED_CROSS);
        else PB_RED_LAUNCH(double, PB_RED_REAL2);
    } else {
        return fail(PB_ERR_INVALID, "bad precision");
    }
#undef PB_RED_LAUNCH
    PB_LAUNCH_CHECK("pb_bin_reduce");
    int per_row = nk * n_ell;
    int total = per_row * n_rows;
    binred_finalize<<<(total + 255) / 256, 256, 0, s>>>(partials, nb, per_row, n_rows, scale, out, accumulate);
    PB_LAUNCH_CHECK("pb_bin_reduce(finalize)");
    return PB_OK;
}

// ------------------------------------------------------------------------------------
// Fisher rows over one k-shell:  out[orow[r]][j] = scale * sum_{i} deg_i Re(conj(F[key_r](m_i)) Q_j(m_i))
// over the shell's mode list m_i.  Chunked: each block stages SR_CH modes of <= SR_R rows
// and SR_CT columns in shared memory, writes one partial per (chunk, row, column);
// a second pass sums the chunks in order.
// ------------------------------------------------------------------------------------
namespace pb {
constexpr int SR_THREADS = 256;
constexpr int SR_CH = 32;   // modes per chunk
constexpr int SR_R = 32;    // rows per launch
constexpr int SR_CT = 32;   // columns per block

struct ShellRowKeys {
    int32_t key[SR_R];
};

template <typename T>
__global__ void __launch_bounds__(SR_THREADS) shell_rows_kernel(Grid g, const typename cplx<T>::type *F,
                                                               const typename cplx<T>::type *Q, int n_rows,
                                                               int n_cols, const int64_t *modes, int64_t n_modes,
                                                               ShellRowKeys keys, double *partials) {
    using C = typename cplx<T>::type;
    __shared__ double2 Fs[SR_R][SR_CH + 1];
    __shared__ double2 Qs[SR_CT][SR_CH + 1];
    const int chunk = blockIdx.x;
    const int j0 = blockIdx.y * SR_CT;
    const int64_t m0 = (int64_t)chunk * SR_CH;
    const int ncols_here = min(SR_CT, n_cols - j0);
    for (int e = threadIdx.x; e < SR_R * SR_CH; e += SR_THREADS) {
        int r = e / SR_CH, i = e - r * SR_CH;
        double2 v = make_double2(0.0, 0.0);
        if (r < n_rows && m0 + i < n_modes) {
            int64_t idx = modes[m0 + i];
            double deg = ((idx % g.nh2) > 0) ? 2.0 : 1.0;
            C f = F[(int64_t)keys.key[r] * g.nhalf + idx];
            v = make_double2(deg * (double)f.x, deg * (double)f.y);
        }
        Fs[r][i] = v;
    }
    for (int e = threadIdx.x; e < SR_CT * SR_CH; e += SR_THREADS) {
        int j = e / SR_CH, i = e - j * SR_CH;
        double2 v = make_double2(0.0, 0.0);
        if (j < ncols_here && m0 + i < n_modes) {
            C q = Q[(int64_t)(j0 + j) * g.nhalf + modes[m0 + i]];
            v = make_double2((double)q.x, (double)q.y);
        }
        Qs[j][i] = v;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < SR_R * SR_CT; o += SR_THREADS) {
        int r = o / SR_CT, j = o - r * SR_CT;
        if (r >= n_rows || j >= ncols_here) continue;
        double s = 0.0;
#pragma unroll 8
        for (int i = 0; i < SR_CH; ++i) s += Fs[r][i].x * Qs[j][i].x + Fs[r][i].y * Qs[j][i].y;
        partials[((int64_t)chunk * n_rows + r) * n_cols + j0 + j] = s;
    }
}

struct ShellRowOut {
    int32_t orow[SR_R];
};

__global__ void shell_rows_finalize(const double *partials, int n_chunks, int n_rows, int n_cols, double scale,
                                    double *out, int64_t out_stride, ShellRowOut o) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_rows * n_cols) return;
    int r = t / n_cols, j = t - r * n_cols;
    double s = 0.0;
    for (int c = 0; c < n_chunks; ++c) s += partials[((int64_t)c * n_rows + r) * n_cols + j];
    out[(int64_t)o.orow[r] * out_stride + j] = s * scale;
}
}  // namespace pb

extern "C" int pb_shell_rows_workspace_size(int64_t n_modes, int n_rows, int n_cols, size_t *bytes) {
    if (!bytes) return fail(PB_ERR_INVALID, "bytes is NULL");
    if (n_modes < 0 || n_rows < 1 || n_rows > SR_R || n_cols < 1)
        return fail(PB_ERR_INVALID, "pb_shell_rows_workspace_size: bad sizes");
    int64_t n_chunks = std::max<int64_t>(1, (n_modes + SR_CH - 1) / SR_CH);
    *bytes = (size_t)n_chunks * n_rows * n_cols * sizeof(double);
    return PB_OK;
}

extern "C" int pb_shell_rows(const pb_grid_t *g, int precision, const void *F, int n_f, const void *Q, int n_cols,
                             const int64_t *modes, int64_t n_modes, const int32_t *row_key, const int32_t *out_row,
                             int n_rows, double scale, double *out, int64_t out_stride, void *workspace,
                             size_t workspace_bytes, void *stream) {
    Grid G;
    int st = make_grid(g, &G);
    if (st) return st;
    if (!F || !Q || !row_key || !out_row || !out) return fail(PB_ERR_INVALID, "pb_shell_rows: NULL argument");
    if (n_rows < 1 || n_rows > SR_R) return fail(PB_ERR_INVALID, "pb_shell_rows: n_rows must be in [1, 32]");
    if (n_cols < 1 || n_f < 1) return fail(PB_ERR_INVALID, "pb_shell_rows: empty input");
    if (n_modes < 0 || (n_modes > 0 && !modes)) return fail(PB_ERR_INVALID, "pb_shell_rows: bad mode list");
    ShellRowKeys keys;
    ShellRowOut orow;
    for (int r = 0; r < SR_R; ++r) {
        keys.key[r] = r < n_rows ? row_key[r] : 0;
        orow.orow[r] = r < n_rows ? out_row[r] : 0;
        if (r < n_rows && (keys.key[r] < 0 || keys.key[r] >= n_f))
            return fail(PB_ERR_INVALID, "pb_shell_rows: row key out of range");
        if (r < n_rows && orow.orow[r] < 0) return fail(PB_ERR_INVALID, "pb_shell_rows: negative output row");
    }
    if (out_stride == 0) out_stride = n_cols;
    int64_t n_chunks = std::max<int64_t>(1, (n_modes + SR_CH - 1) / SR_CH);
    size_t need = (size_t)n_chunks * n_rows * n_cols * sizeof(double);
    if (!workspace || workspace_bytes < need) return fail(PB_ERR_WORKSPACE, "pb_shell_rows: workspace too small");
    if (n_chunks > 2147483647) return fail(PB_ERR_INVALID, "pb_shell_rows: too many modes");
    cudaStream_t s = as_stream(stream);
    dim3 grid((unsigned)n_chunks, (n_cols + SR_CT - 1) / SR_CT);
    double *partials = (double *)workspace;
    if (n_modes == 0) {
        // empty shell: zero partials through a one-chunk launch with no modes
    }
    if (precision == PB_F64)
        shell_rows_kernel<double><<<grid, SR_THREADS, 0, s>>>(G, (const double2 *)F, (const double2 *)Q, n_rows,
                                                              n_cols, modes, n_modes, keys, partials);
    else if (precision == PB_F32)
        shell_rows_kernel<float><<<grid, SR_THREADS, 0, s>>>(G, (const float2 *)F, (const float2 *)Q, n_rows, n_cols,
                                                             modes, n_modes, keys, partials);
    else
        return fail(PB_ERR_INVALID, "bad precision");
    PB_LAUNCH_CHECK("pb_shell_rows");
    int total = n_rows * n_cols;
    shell_rows_finalize<<<(total + 255) / 256, 256, 0, s>>>(partials, (int)n_chunks, n_rows, n_cols, scale, out,
                                                           out_stride, orow);
    PB_LAUNCH_CHECK("pb_shell_rows(finalize)");
    return PB_OK;
}

// ------------------------------------------------------------------------------------
// pb_bin_reduce_noalloc: the k-bin reduction with its scratch in a fixed device array.
//
// Some callers cannot hand this library a workspace: a binding that only forwards the
// input and output pointers it was given and owns no device allocator, or a host program
// whose GPU memory is entirely reserved by another framework's pool, where a cudaMalloc
// (which may also synchronise the device) is not acceptable.  For them the per-block
// partial sums live in the file-scope array below, PB_BIN_REDUCE_NOALLOC_MAX_DOUBLES
// doubles (2 MiB); every GPU that loads the library keeps it until the process exits.
//
// The array's host-side name is only a stand-in for the device symbol, so its device
// address is looked up once per device with cudaGetSymbolAddress, with that device
// current, on the first call made on that device; make that first call before any stream
// capture.  The address is kept for the life of the process: a program that resets the
// device (cudaDeviceReset) must not call this entry point afterwards.  All calls share the
// one array: calls whose kernels overlap on the GPU (other streams, other host threads)
// race on it and must be serialised by the caller.  Each call writes every partial it later
// reads, so nothing is carried over from the previous call.  Spectra go through the same
// deterministic multi-row kernel as pb_bin_reduce, with as many blocks per row as fit.
// ------------------------------------------------------------------------------------
#include <mutex>

namespace pb {
static __device__ __align__(256) double g_binred_scratch[PB_BIN_REDUCE_NOALLOC_MAX_DOUBLES];

static std::mutex g_binred_scratch_mu;
static double *g_binred_scratch_dev[64];  // device address per device ordinal, looked up once

static int binred_scratch_address(double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_check(e, "pb_bin_reduce_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= 64) return fail(PB_ERR_UNSUPPORTED, "pb_bin_reduce_noalloc: device ordinal >= 64");
    std::lock_guard<std::mutex> lock(g_binred_scratch_mu);
    if (!g_binred_scratch_dev[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_binred_scratch);
        if (e != cudaSuccess) return cuda_check(e, "pb_bin_reduce_noalloc: cudaGetSymbolAddress");
        g_binred_scratch_dev[dev] = (double *)p;
    }
    *out = g_binred_scratch_dev[dev];
    return PB_OK;
}
}  // namespace pb

extern "C" int pb_bin_reduce_noalloc(const pb_grid_t *g, int precision, int mode, const void *a, const void *b,
                                     int n_rows, int64_t row_stride, const double *edges, int nk,
                                     const int32_t *ells, int n_ell, double scale, double *out, int accumulate,
                                     void *stream) {
    Grid G;
    int st = make_grid(g, &G);
    if (st) return st;
    if (nk < 1 || nk > PB_RED_MAX_BINS) return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: nk must be in [1, 64]");
    if (n_ell < 1 || n_ell > PB_RED_MAX_ELLS)
        return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: n_ell must be in [1, 9]");
    if (n_rows < 1 || n_rows > 65535)
        return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: n_rows must be in [1, 65535]");
    if (!edges || !ells || !out) return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: NULL argument");
    if (mode == PB_RED_ABS2 && !a) return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: ABS2 needs a");
    if (mode == PB_RED_CROSS && (!a || !b)) return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: CROSS needs a and b");
    if (mode < 0 || mode > 2) return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: bad mode");
    if (precision != PB_F32 && precision != PB_F64) return fail(PB_ERR_INVALID, "bad precision");
    // partial sums: one slot of n_ell*nk doubles per (row, block); shrink the block count
    // to fit the fixed array, down to one block per row
    const int64_t per_row_block = (int64_t)nk * n_ell;
    const int64_t fit = PB_BIN_REDUCE_NOALLOC_MAX_DOUBLES / ((int64_t)n_rows * per_row_block);
    if (fit < 1)
        return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: n_rows * nk * n_ell = " +
                                        std::to_string((int64_t)n_rows * per_row_block) +
                                        " doubles exceeds the fixed scratch of " +
                                        std::to_string((int64_t)PB_BIN_REDUCE_NOALLOC_MAX_DOUBLES) +
                                        "; use pb_bin_reduce with a workspace");
    if (row_stride == 0) row_stride = G.nhalf;
    RedParams p;
    for (int i = 0; i <= nk; ++i) {
        p.edges[i] = edges[i];
        if (i > 0 && !(edges[i] > edges[i - 1]))
            return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: bin edges must be strictly increasing");
    }
    for (int e = 0; e < n_ell; ++e) {
        if (ells[2 * e] < 0 || ells[2 * e] > 4 || ells[2 * e + 1] < 0 || ells[2 * e + 1] > 4)
            return fail(PB_ERR_INVALID, "pb_bin_reduce_noalloc: Legendre order must be in [0, 4]");
        p.la[e] = (int8_t)ells[2 * e];
        p.lb[e] = (int8_t)ells[2 * e + 1];
    }
    p.nk = nk;
    p.n_ell = n_ell;
    double *partials = nullptr;
    st = binred_scratch_address(&partials);
    if (st) return st;
    int nb = (int)std::min<int64_t>(red_blocks(G), fit);
    cudaStream_t s = as_stream(stream);
    if (mode != PB_RED_REAL2) {
        // spectra: the deterministic multi-row kernel of pb_bin_reduce (its accumulators are
        // dynamic shared memory, not device memory), on the block count that fits the array
        const int per = nk * n_ell;
        const int rpg = std::max(1, std::min(n_rows, RR_ACC_DOUBLES / per));
        const size_t smem = rr_acc_len(rpg, n_ell, nk) * sizeof(double) + (size_t)n_ell * RR_TILE * sizeof(double) +
                            (size_t)RR_TILE * (sizeof(double2) + sizeof(int));
        dim3 rgrid(nb, (n_rows + rpg - 1) / rpg);
#define PB_RR_LAUNCH(T, M)                                                                                   \
    do {                                                                                                     \
        PB_CUDA(cudaFuncSetAttribute(binred_rows_kernel<T, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                     (int)smem));                                                            \
        binred_rows_kernel<T, M><<<rgrid, RED_THREADS, smem, s>>>(G, (const cplx<T>::type *)a,              \
                                                                  (const cplx<T>::type *)b, row_stride, p,   \
                                                                  n_rows, rpg, partials);                    \
    } while (0)
        if (precision == PB_F32) {
            if (mode == PB_RED_ABS2) PB_RR_LAUNCH(float, PB_RED_ABS2);
            else PB_RR_LAUNCH(float, PB_RED_CROSS);
        } else {
            if (mode == PB_RED_ABS2) PB_RR_LAUNCH(double, PB_RED_ABS2);
            else PB_RR_LAUNCH(double, PB_RED_CROSS);
        }
#undef PB_RR_LAUNCH
    } else {
        dim3 grid(nb, n_rows);
        if (precision == PB_F32)
            binred_kernel<float, PB_RED_REAL2><<<grid, RED_THREADS, 0, s>>>(G, nullptr, nullptr, (const float *)a,
                                                                            row_stride, p, partials);
        else
            binred_kernel<double, PB_RED_REAL2><<<grid, RED_THREADS, 0, s>>>(G, nullptr, nullptr, (const double *)a,
                                                                             row_stride, p, partials);
    }
    PB_LAUNCH_CHECK("pb_bin_reduce_noalloc");
    int per_row = nk * n_ell;
    int total = per_row * n_rows;
    binred_finalize<<<(total + 255) / 256, 256, 0, s>>>(partials, nb, per_row, n_rows, scale, out, accumulate);
    PB_LAUNCH_CHECK("pb_bin_reduce_noalloc(finalize)");
    return PB_OK;
}
