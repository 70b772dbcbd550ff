// Core entry points: errors, cuFFT plans, the spectral filter, elementwise products
// and the Gaussian-random-field kernel.
#include <cufft.h>
#include <algorithm>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>
#include "pb_common.cuh"

namespace pb {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    set_error(msg);
    return code;
}

int cuda_check(cudaError_t e, const char *where) {
    return fail(PB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

static thread_local pb_tuning_t g_tuning = {0, 0, 0, 0, 0, 0, 0, 0};

const pb_tuning_t &tuning() { return g_tuning; }

int num_sms() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    return n > 0 ? n : 148;
}

int make_grid(const pb_grid_t *g, Grid *out) {
    if (!g) return fail(PB_ERR_INVALID, "grid is NULL");
    for (int i = 0; i < 3; ++i) {
        if (g->n[i] <= 0) return fail(PB_ERR_INVALID, "grid dimensions must be positive");
        if (!(g->kf[i] > 0.0)) return fail(PB_ERR_INVALID, "fundamental frequencies must be positive");
    }
    if (g->n[2] % 2 != 0)
        return fail(PB_ERR_INVALID, "Last dimension of grid must be even for real-to-complex FFTs.");
    out->n0 = g->n[0];
    out->n1 = g->n[1];
    out->n2 = g->n[2];
    out->nh2 = g->n[2] / 2 + 1;
    out->kf0 = g->kf[0];
    out->kf1 = g->kf[1];
    out->kf2 = g->kf[2];
    out->los = (g->flags & PB_GRID_LOS) ? 1 : 0;
    out->l0 = out->los ? g->los[0] : 0.0;
    out->l1 = out->los ? g->los[1] : 0.0;
    out->l2 = out->los ? g->los[2] : 1.0;
    if (out->los && !(out->l0 * out->l0 + out->l1 * out->l1 + out->l2 * out->l2 > 0.0))
        return fail(PB_ERR_INVALID, "line of sight must be a non-zero vector");
    out->nhalf = (int64_t)out->n0 * out->n1 * out->nh2;
    out->nreal = (int64_t)out->n0 * out->n1 * out->n2;
    return PB_OK;
}

static int grid_blocks(int64_t work, int threads, int per_sm = 8) {
    int64_t b = (work + threads - 1) / threads;
    int64_t cap = (int64_t)num_sms() * per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

// ------------------------------------------------------------------------------------
// spectral filter
// ------------------------------------------------------------------------------------
struct FilterParams {
    double lo[PB_FILTER_MAX_MAPS];
    double hi[PB_FILTER_MAX_MAPS];
    double scale[PB_FILTER_MAX_MAPS];
    int32_t src[PB_FILTER_MAX_MAPS];
    int16_t dst[PB_FILTER_MAX_MAPS];
    int8_t l1[PB_FILTER_MAX_MAPS];
    int8_t l2[PB_FILTER_MAX_MAPS];
    int8_t wpow[PB_FILTER_MAX_MAPS];
    int32_t n_maps;
};

template <typename T>
__global__ void __launch_bounds__(256) filter_kernel(Grid g, Grid go, const typename cplx<T>::type *src,
                                                     int64_t src_stride, typename cplx<T>::type *out, const T *w,
                                                     int acc, FilterParams p) {
    // iterate over the modes of the output grid `go`; each reads the source mode of the
    // same frequency on `g` (identical when the grids agree; a frequency the source grid
    // does not hold reads 0)
    using C = typename cplx<T>::type;
    const bool same = (go.n0 == g.n0 && go.n1 == g.n1 && go.n2 == g.n2);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < go.nhalf; idx += stride) {
        Mode md = mode_of(go, idx);
        int64_t sidx = idx;
        bool have = true;
        if (!same) {
            int l = (int)(idx % go.nh2);
            int64_t r = idx / go.nh2;
            int j = (int)(r % go.n1);
            int i = (int)(r / go.n1);
            int fi = freq_index(i, go.n0), fj = freq_index(j, go.n1);
            have = (2 * fi >= -g.n0) && (2 * fi < g.n0) && (2 * fj >= -g.n1) && (2 * fj < g.n1) && (l < g.nh2);
            int si = fi < 0 ? fi + g.n0 : fi, sj = fj < 0 ? fj + g.n1 : fj;
            sidx = have ? ((int64_t)si * g.n1 + sj) * g.nh2 + l : 0;
        }
        double wv = (w && have) ? (double)w[sidx] : 1.0;
        int cached = -1;
        C s;
        s.x = 1;
        s.y = 0;
        for (int m = 0; m < p.n_maps; ++m) {
            C *o = out + (int64_t)p.dst[m] * go.nhalf + idx;
            bool in = (p.lo[m] <= md.k) && (md.k < p.hi[m]);
            if (!in) {
                if (!acc) { C z; z.x = 0; z.y = 0; *o = z; }
                continue;
            }
            if (src && p.src[m] != cached) {
                if (have) {
                    s = src[(int64_t)p.src[m] * src_stride + sidx];
                } else {
                    s.x = 0;
                    s.y = 0;
                }
                cached = p.src[m];
            }
            double f = p.scale[m] * legendre(p.l1[m], md.mu) * legendre(p.l2[m], md.mu);
            if (p.wpow[m] == 1) f *= wv;
            else if (p.wpow[m] == 2) f *= wv * wv;
            else if (p.wpow[m] == -1) f = (wv != 0.0) ? f / wv : 0.0;
            C v;
            v.x = (T)((double)s.x * f);
            v.y = (T)((double)s.y * f);
            if (acc) {
                C prev = *o;
                v.x += prev.x;
                v.y += prev.y;
            }
            *o = v;
        }
    }
}

// ------------------------------------------------------------------------------------
// binned-weight filter: out(k) = scale * src(k) * w(k)^wpow * sum_e coef[e][bin(k)] L_{ells[e]}(mu)
// ------------------------------------------------------------------------------------
struct BinWParams {
    double edges[PB_RED_MAX_BINS + 1];
    int8_t ell[PB_RED_MAX_ELLS];
    int32_t nk, n_ell, wpow;
    double scale;
};

template <typename T>
__global__ void binned_filter_kernel(Grid g, const typename cplx<T>::type *src, typename cplx<T>::type *out,
                                     const double *coef, const T *w, BinWParams p) {
    using C = typename cplx<T>::type;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < g.nhalf; idx += stride) {
        Mode md = mode_of(g, idx);
        int b = -1;
        if (p.edges[0] <= md.k && md.k < p.edges[p.nk]) {
            int lo = 0, hi = p.nk;
            while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (p.edges[mid] <= md.k) lo = mid;
                else hi = mid;
            }
            b = lo;
        }
        C v;
        v.x = 0;
        v.y = 0;
        if (b >= 0) {
            double f = 0.0;
            for (int e = 0; e < p.n_ell; ++e) f += coef[e * p.nk + b] * legendre(p.ell[e], md.mu);
            f *= p.scale;
            if (w) {
                double wv = (double)w[idx];
                if (p.wpow == 1) f *= wv;
                else if (p.wpow == 2) f *= wv * wv;
                else if (p.wpow == -1) f = wv != 0.0 ? f / wv : 0.0;
                else if (p.wpow == -2) f = wv != 0.0 ? f / (wv * wv) : 0.0;
            }
            C s = src[idx];
            v.x = (T)((double)s.x * f);
            v.y = (T)((double)s.y * f);
        }
        out[idx] = v;
    }
}

}  // namespace pb

using namespace pb;

// ------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------
extern "C" int pb_abi_version(void) { return PB_ABI_VERSION; }

extern "C" const char *pb_last_error(void) { return g_last_error.c_str(); }

extern "C" int pb_set_tuning(const pb_tuning_t *t) {
    if (!t) {
        g_tuning = pb_tuning_t{0, 0, 0, 0, 0, 0, 0, 0};
        return PB_OK;
    }
    if (t->tc_tile != 0 && t->tc_tile != 32 && t->tc_tile != 64 && t->tc_tile != 128)
        return fail(PB_ERR_INVALID, "pb_set_tuning: tc_tile must be 0, 32, 64 or 128");
    if (t->tc_stages != 0 && (t->tc_stages < 2 || t->tc_stages > 6))
        return fail(PB_ERR_INVALID, "pb_set_tuning: tc_stages must be 0 or in [2, 6]");
    if (t->tc_chain != 0 && t->tc_chain != 256 && t->tc_chain != 512 && t->tc_chain != 1024 && t->tc_chain != 2048)
        return fail(PB_ERR_INVALID, "pb_set_tuning: tc_chain must be 0, 256, 512, 1024 or 2048");
    if (t->red_method < 0 || t->red_method > 2) return fail(PB_ERR_INVALID, "pb_set_tuning: red_method in [0, 2]");
    if (t->red_warps < 0 || t->red_warps > 8) return fail(PB_ERR_INVALID, "pb_set_tuning: red_warps in [0, 8]");
    if (t->red_waves < 0 || t->red_waves > 32) return fail(PB_ERR_INVALID, "pb_set_tuning: red_waves in [0, 32]");
    if (t->tc_wait < 0 || t->tc_wait > 2) return fail(PB_ERR_INVALID, "pb_set_tuning: tc_wait in [0, 2]");
    if (t->tc_dsets < 0 || t->tc_dsets > 2) return fail(PB_ERR_INVALID, "pb_set_tuning: tc_dsets in [0, 2]");
    g_tuning = *t;
    return PB_OK;
}

extern "C" int pb_get_tuning(pb_tuning_t *t) {
    if (!t) return fail(PB_ERR_INVALID, "pb_get_tuning: NULL");
    *t = g_tuning;
    return PB_OK;
}

struct pb_fft_plan {
    cufftHandle h;
    int direction;
    int precision;
    size_t ws;
};

static const char *cufft_name(cufftResult r) {
    switch (r) {
        case CUFFT_SUCCESS: return "CUFFT_SUCCESS";
        case CUFFT_INVALID_PLAN: return "CUFFT_INVALID_PLAN";
        case CUFFT_ALLOC_FAILED: return "CUFFT_ALLOC_FAILED";
        case CUFFT_INVALID_VALUE: return "CUFFT_INVALID_VALUE";
        case CUFFT_INTERNAL_ERROR: return "CUFFT_INTERNAL_ERROR";
        case CUFFT_EXEC_FAILED: return "CUFFT_EXEC_FAILED";
        case CUFFT_SETUP_FAILED: return "CUFFT_SETUP_FAILED";
        case CUFFT_INVALID_SIZE: return "CUFFT_INVALID_SIZE";
        default: return "CUFFT_ERROR";
    }
}

// a failed cuFFT call reports the CUDA runtime's pending error too (a launch failure such as
// out-of-resources shows up there)
#define PB_CUFFT(call)                                                                 \
    do {                                                                               \
        cufftResult _r = (call);                                                       \
        if (_r != CUFFT_SUCCESS) {                                                     \
            cudaError_t _e = cudaGetLastError();                                       \
            return fail(PB_ERR_CUFFT, std::string(#call ": ") + cufft_name(_r) +      \
                                          (_e != cudaSuccess ? std::string(" (CUDA: ") + cudaGetErrorString(_e) + ")" \
                                                             : std::string()));        \
        }                                                                              \
    } while (0)

extern "C" int pb_fft_plan_create(const pb_grid_t *g, int batch, int precision, int direction,
                                  pb_fft_plan **plan, size_t *workspace_bytes) {
    Grid G;
    int st = make_grid(g, &G);
    if (st) return st;
    if (!plan) return fail(PB_ERR_INVALID, "plan out-pointer is NULL");
    if (batch < 1) return fail(PB_ERR_INVALID, "batch must be >= 1");
    if (precision != PB_F32 && precision != PB_F64) return fail(PB_ERR_INVALID, "bad precision");
    if (direction != PB_FFT_R2C && direction != PB_FFT_C2R) return fail(PB_ERR_INVALID, "bad direction");
    cufftType type = direction == PB_FFT_R2C ? (precision == PB_F64 ? CUFFT_D2Z : CUFFT_R2C)
                                             : (precision == PB_F64 ? CUFFT_Z2D : CUFFT_C2R);
    long long n[3] = {G.n0, G.n1, G.n2};
    long long rdist = G.nreal, cdist = G.nhalf;
    long long idist = direction == PB_FFT_R2C ? rdist : cdist;
    long long odist = direction == PB_FFT_R2C ? cdist : rdist;
    pb_fft_plan *p = new pb_fft_plan();
    p->direction = direction;
    p->precision = precision;
    cufftResult r = cufftCreate(&p->h);
    if (r != CUFFT_SUCCESS) {
        delete p;
        return fail(PB_ERR_CUFFT, std::string("cufftCreate: ") + cufft_name(r));
    }
    r = cufftSetAutoAllocation(p->h, 0);
    size_t ws = 0;
    if (r == CUFFT_SUCCESS)
        r = cufftMakePlanMany64(p->h, 3, n, nullptr, 1, idist, nullptr, 1, odist, type, batch, &ws);
    if (r != CUFFT_SUCCESS) {
        cufftDestroy(p->h);
        delete p;
        return fail(PB_ERR_CUFFT, std::string("cufftMakePlanMany64: ") + cufft_name(r));
    }
    p->ws = ws;
    *plan = p;
    if (workspace_bytes) *workspace_bytes = ws;
    return PB_OK;
}

extern "C" int pb_fft_exec(pb_fft_plan *p, const void *in, void *out, void *workspace, void *stream) {
    if (!p || !in || !out) return fail(PB_ERR_INVALID, "pb_fft_exec: NULL argument");
    if (p->ws && !workspace) return fail(PB_ERR_WORKSPACE, "pb_fft_exec: plan needs a workspace");
    {
        // an error left pending by earlier work on this thread would otherwise surface as a
        // failure of this transform
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_check(e, "pb_fft_exec (error pending before the transform)");
    }
    PB_CUFFT(cufftSetStream(p->h, as_stream(stream)));
    if (p->ws) PB_CUFFT(cufftSetWorkArea(p->h, workspace));
    void *i = const_cast<void *>(in);
    if (p->direction == PB_FFT_R2C) {
        if (p->precision == PB_F64)
            PB_CUFFT(cufftExecD2Z(p->h, (cufftDoubleReal *)i, (cufftDoubleComplex *)out));
        else
            PB_CUFFT(cufftExecR2C(p->h, (cufftReal *)i, (cufftComplex *)out));
    } else {
        if (p->precision == PB_F64)
            PB_CUFFT(cufftExecZ2D(p->h, (cufftDoubleComplex *)i, (cufftDoubleReal *)out));
        else
            PB_CUFFT(cufftExecC2R(p->h, (cufftComplex *)i, (cufftReal *)out));
    }
    return PB_OK;
}

extern "C" int pb_fft_plan_destroy(pb_fft_plan *p) {
    if (!p) return PB_OK;
    cufftResult r = cufftDestroy(p->h);
    delete p;
    if (r != CUFFT_SUCCESS) return fail(PB_ERR_CUFFT, std::string("cufftDestroy: ") + cufft_name(r));
    return PB_OK;
}

extern "C" int pb_spectral_filter(const pb_grid_t *g, const int32_t *out_n, int precision, const void *src,
                                  int64_t src_stride, void *out, int n_maps, const int32_t *src_idx,
                                  const int32_t *dst_idx, const double *lo, const double *hi, const int32_t *l1,
                                  const int32_t *l2, const double *scale, const int32_t *wpow, const void *w,
                                  int accumulate, void *stream) {
    Grid G, GO;
    int st = make_grid(g, &G);
    if (st) return st;
    GO = G;
    if (out_n) {
        pb_grid_t go = *g;
        for (int i = 0; i < 3; ++i) go.n[i] = out_n[i];
        st = make_grid(&go, &GO);
        if (st) return st;
        if (w && (GO.n0 > G.n0 || GO.n1 > G.n1 || GO.n2 > G.n2))
            return fail(PB_ERR_INVALID, "pb_spectral_filter: a weight grid needs an output grid no larger than the input");
    }
    if (!out) return fail(PB_ERR_INVALID, "pb_spectral_filter: out is NULL");
    if (n_maps < 1 || n_maps > PB_FILTER_MAX_MAPS)
        return fail(PB_ERR_INVALID, "pb_spectral_filter: n_maps must be in [1, 128]");
    if (!lo || !hi || !l1 || !l2 || !scale)
        return fail(PB_ERR_INVALID, "pb_spectral_filter: NULL parameter array");
    FilterParams p;
    p.n_maps = n_maps;
    for (int m = 0; m < n_maps; ++m) {
        if (l1[m] < 0 || l1[m] > 4 || l2[m] < 0 || l2[m] > 4)
            return fail(PB_ERR_INVALID, "pb_spectral_filter: Legendre order must be in [0, 4]");
        int wp = wpow ? wpow[m] : 0;
        if (wp < -1 || wp > 2) return fail(PB_ERR_INVALID, "pb_spectral_filter: wpow must be -1, 0, 1 or 2");
        if (wp != 0 && !w) return fail(PB_ERR_INVALID, "pb_spectral_filter: wpow set but weight grid is NULL");
        p.lo[m] = lo[m];
        p.hi[m] = hi[m];
        p.scale[m] = scale[m];
        p.src[m] = src_idx ? src_idx[m] : 0;
        if (p.src[m] < 0) return fail(PB_ERR_INVALID, "pb_spectral_filter: negative source index");
        int d = dst_idx ? dst_idx[m] : m;
        if (d < 0 || d > 32767) return fail(PB_ERR_INVALID, "pb_spectral_filter: output index out of range");
        if (dst_idx && !accumulate)
            return fail(PB_ERR_INVALID, "pb_spectral_filter: an output index map needs accumulate (outputs may repeat)");
        p.dst[m] = (int16_t)d;
        p.l1[m] = (int8_t)l1[m];
        p.l2[m] = (int8_t)l2[m];
        p.wpow[m] = (int8_t)wp;
    }
    int threads = 256;
    int blocks = grid_blocks(GO.nhalf, threads);
    if (precision == PB_F32)
        filter_kernel<float><<<blocks, threads, 0, as_stream(stream)>>>(
            G, GO, (const float2 *)src, src_stride, (float2 *)out, (const float *)w, accumulate, p);
    else if (precision == PB_F64)
        filter_kernel<double><<<blocks, threads, 0, as_stream(stream)>>>(
            G, GO, (const double2 *)src, src_stride, (double2 *)out, (const double *)w, accumulate, p);
    else
        return fail(PB_ERR_INVALID, "bad precision");
    PB_LAUNCH_CHECK("pb_spectral_filter");
    return PB_OK;
}

// ------------------------------------------------------------------------------------
// elementwise
// ------------------------------------------------------------------------------------
template <typename T>
__global__ void ew_kernel(int op, int64_t n, const T *x, const T *y, int64_t y_period, const T *z, const T *u, T s,
                          T *out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        T v;
        T yv = y[y_period ? i % y_period : i];
        if (op == PB_EW_MUL) v = x[i] * yv;
        else v = x[i] * yv - z[i] * u[i];
        out[i] = s * v;
    }
}

// FP32 -> FP64, exact: four values per step (one 16-byte read, two 16-byte writes) when both
// arrays are 16-byte aligned, then the tail
__global__ void widen_kernel(int64_t n, const float *x, double *out, int vec) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t done = 0;
    if (vec) {
        const int64_t n4 = n >> 2;
        for (int64_t q = i; q < n4; q += stride) {
            const float4 v = reinterpret_cast<const float4 *>(x)[q];
            reinterpret_cast<double2 *>(out)[2 * q] = make_double2(v.x, v.y);
            reinterpret_cast<double2 *>(out)[2 * q + 1] = make_double2(v.z, v.w);
        }
        done = n4 << 2;
    }
    for (int64_t k = done + i; k < n; k += stride) out[k] = (double)x[k];
}

extern "C" int pb_elementwise(int precision, int op, int64_t n, const void *x, const void *y, int64_t y_period,
                              const void *z, const void *u, double s, void *out, void *stream) {
    if (n < 0) return fail(PB_ERR_INVALID, "pb_elementwise: negative size");
    if (n == 0) return PB_OK;
    if (op == PB_EW_WIDEN) {
        if (!x || !out) return fail(PB_ERR_INVALID, "pb_elementwise: NULL argument");
        if (precision != PB_F32) return fail(PB_ERR_INVALID, "pb_elementwise: WIDEN reads FP32 (precision PB_F32)");
        const int vec = (((uintptr_t)x | (uintptr_t)out) & 15) == 0;
        const int threads = 256;
        widen_kernel<<<grid_blocks(vec ? (n + 3) / 4 : n, threads, 16), threads, 0, as_stream(stream)>>>(
            n, (const float *)x, (double *)out, vec);
        PB_LAUNCH_CHECK("pb_elementwise");
        return PB_OK;
    }
    if (!x || !y || !out) return fail(PB_ERR_INVALID, "pb_elementwise: NULL argument");
    if (op == PB_EW_PRODDIFF && (!z || !u)) return fail(PB_ERR_INVALID, "pb_elementwise: PRODDIFF needs z, u");
    if (op != PB_EW_MUL && op != PB_EW_PRODDIFF) return fail(PB_ERR_INVALID, "pb_elementwise: bad op");
    if (y_period < 0 || (y_period > 0 && n % y_period != 0))
        return fail(PB_ERR_INVALID, "pb_elementwise: y_period must divide n");
    if (op == PB_EW_PRODDIFF && y_period != 0) return fail(PB_ERR_INVALID, "pb_elementwise: PRODDIFF takes no y_period");
    int threads = 256;
    int blocks = grid_blocks(n, threads, 16);
    if (precision == PB_F32)
        ew_kernel<float><<<blocks, threads, 0, as_stream(stream)>>>(op, n, (const float *)x, (const float *)y, y_period,
                                                                   (const float *)z, (const float *)u,
                                                                   (float)s, (float *)out);
    else if (precision == PB_F64)
        ew_kernel<double><<<blocks, threads, 0, as_stream(stream)>>>(op, n, (const double *)x, (const double *)y, y_period,
                                                                    (const double *)z, (const double *)u, s,
                                                                    (double *)out);
    else
        return fail(PB_ERR_INVALID, "bad precision");
    PB_LAUNCH_CHECK("pb_elementwise");
    return PB_OK;
}

// ------------------------------------------------------------------------------------
// Gaussian random field from white noise
// ------------------------------------------------------------------------------------
template <typename T>
__global__ void grf_kernel(Grid g, const double *nre, const double *nim, int n_batch, const double *amp,
                           double scale, typename cplx<T>::type *out) {
    using C = typename cplx<T>::type;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t total = g.nhalf * n_batch;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        int64_t bidx = t / g.nhalf;
        int64_t idx = t - bidx * g.nhalf;
        int l = (int)(idx % g.nh2);
        int64_t r = idx / g.nh2;
        int j = (int)(r % g.n1);
        int i = (int)(r / g.n1);
        int mi = (g.n0 - i) % g.n0, mj = (g.n1 - j) % g.n1, ml = (g.n2 - l) % g.n2;
        const double *re = nre + bidx * g.nreal;
        const double *im = nim + bidx * g.nreal;
        int64_t p = ((int64_t)i * g.n1 + j) * g.n2 + l;
        int64_t q = ((int64_t)mi * g.n1 + mj) * g.n2 + ml;
        double ar = 0.0, ai = 0.0;
        if (p != 0) {  // r[0,0,0] = 0 and its mirror is itself
            ar = 0.5 * (re[p] + re[q]);
            ai = 0.5 * (im[p] - im[q]);
        }
        double a = amp[idx];
        C v;
        v.x = (T)(ar * a * scale);
        v.y = (T)(ai * a * scale);
        out[t] = v;
    }
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): ten rounds of two 32x32->64 multiplies with the published multipliers, the key
// bumped by the Weyl constants between rounds.
struct Philox4 {
    uint32_t x[4];
};

__device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                                 uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = M0 * c0, hi0 = __umulhi(M0, c0);
        const uint32_t lo1 = M1 * c2, hi1 = __umulhi(M1, c2);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0;
        c1 = n1;
        c2 = n2;
        c3 = n3;
        k0 += W0;
        k1 += W1;
    }
    Philox4 o;
    o.x[0] = c0;
    o.x[1] = c1;
    o.x[2] = c2;
    o.x[3] = c3;
    return o;
}

// (re, im) white noise at full-grid voxel p of the field with this seed: Box-Muller on
// u1 = (x0 + 1/2) 2^-32, u2 = (x1 + 1/2) 2^-32 (both in (0, 1))
__device__ __forceinline__ void philox_noise(int64_t seed, int64_t p, double &re, double &im) {
    Philox4 r = philox4x32_10((uint32_t)p, (uint32_t)((uint64_t)p >> 32), PB_PHILOX_DOMAIN, 0u, (uint32_t)seed,
                              (uint32_t)((uint64_t)seed >> 32));
    const double u1 = ((double)r.x[0] + 0.5) * 2.3283064365386963e-10;
    const double u2 = ((double)r.x[1] + 0.5) * 2.3283064365386963e-10;
    const double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    re = rad * c;
    im = rad * s;
}

template <typename T>
__global__ void grf_philox_kernel(Grid g, const int64_t *seeds, int n_batch, const double *amp, double scale,
                                  typename cplx<T>::type *out) {
    using C = typename cplx<T>::type;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t total = g.nhalf * n_batch;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        int64_t bidx = t / g.nhalf;
        int64_t idx = t - bidx * g.nhalf;
        int l = (int)(idx % g.nh2);
        int64_t r = idx / g.nh2;
        int j = (int)(r % g.n1);
        int i = (int)(r / g.n1);
        int mi = (g.n0 - i) % g.n0, mj = (g.n1 - j) % g.n1, ml = (g.n2 - l) % g.n2;
        int64_t p = ((int64_t)i * g.n1 + j) * g.n2 + l;
        int64_t q = ((int64_t)mi * g.n1 + mj) * g.n2 + ml;
        double ar = 0.0, ai = 0.0;
        if (p != 0) {
            const int64_t seed = seeds[bidx];
            double pr, pi, qr, qi;
            philox_noise(seed, p, pr, pi);
            philox_noise(seed, q, qr, qi);
            ar = 0.5 * (pr + qr);
            ai = 0.5 * (pi - qi);
        }
        double a = amp[idx];
        C v;
        v.x = (T)(ar * a * scale);
        v.y = (T)(ai * a * scale);
        out[t] = v;
    }
}

extern "C" int pb_grf_philox(const pb_grid_t *g, int precision, const int64_t *seeds, int n_batch, const double *amp,
                             double scale, void *out, void *stream) {
    Grid G;
    int st = make_grid(g, &G);
    if (st) return st;
    if (!seeds || !amp || !out) return fail(PB_ERR_INVALID, "pb_grf_philox: NULL argument");
    if (n_batch < 1) return fail(PB_ERR_INVALID, "pb_grf_philox: n_batch must be >= 1");
    int threads = 256;
    int blocks = grid_blocks(G.nhalf * n_batch, threads, 16);
    if (precision == PB_F32)
        grf_philox_kernel<float><<<blocks, threads, 0, as_stream(stream)>>>(G, seeds, n_batch, amp, scale,
                                                                           (float2 *)out);
    else if (precision == PB_F64)
        grf_philox_kernel<double><<<blocks, threads, 0, as_stream(stream)>>>(G, seeds, n_batch, amp, scale,
                                                                            (double2 *)out);
    else
        return fail(PB_ERR_INVALID, "bad precision");
    PB_LAUNCH_CHECK("pb_grf_philox");
    return PB_OK;
}

extern "C" int pb_grf_from_noise(const pb_grid_t *g, int precision, const double *noise_re, const double *noise_im,
                                 int n_batch, const double *amp, double scale, void *out, void *stream) {
    Grid G;
    int st = make_grid(g, &G);
    if (st) return st;
    if (!noise_re || !noise_im || !amp || !out) return fail(PB_ERR_INVALID, "pb_grf_from_noise: NULL argument");
    if (n_batch < 1) return fail(PB_ERR_INVALID, "pb_grf_from_noise: n_batch must be >= 1");
    int threads = 256;
    int blocks = grid_blocks(G.nhalf * n_batch, threads, 16);
    if (precision == PB_F32)
        grf_kernel<float><<<blocks, threads, 0, as_stream(stream)>>>(G, noise_re, noise_im, n_batch, amp, scale,
                                                                    (float2 *)out);
    else if (precision == PB_F64)
        grf_kernel<double><<<blocks, threads, 0, as_stream(stream)>>>(G, noise_re, noise_im, n_batch, amp, scale,
                                                                     (double2 *)out);
    else
        return fail(PB_ERR_INVALID, "bad precision");
    PB_LAUNCH_CHECK("pb_grf_from_noise");
    return PB_OK;
}

// ------------------------------------------------------------------------------------
// batched pair products  out[p] = s * (X[i_p] * Y[j_p] - Z[i_p] * U[j_p])
// ------------------------------------------------------------------------------------
namespace pb {
struct PairParams {
    int32_t i[PB_PAIR_MAX];
    int32_t j[PB_PAIR_MAX];
    int32_t n;
};

template <typename T>
__global__ void pair_kernel(int64_t n_vox, const T *X, const T *Y, const T *Z, const T *U, T s, T *out,
                            PairParams p) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int pidx = blockIdx.y;
    const T *x = X + (int64_t)p.i[pidx] * n_vox;
    const T *y = Y + (int64_t)p.j[pidx] * n_vox;
    const T *z = Z ? Z + (int64_t)p.i[pidx] * n_vox : nullptr;
    const T *u = U ? U + (int64_t)p.j[pidx] * n_vox : nullptr;
    T *o = out + (int64_t)pidx * n_vox;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_vox; v += stride) {
        T r = x[v] * y[v];
        if (z) r -= z[v] * u[v];
        o[v] = s * r;
    }
}
}  // namespace pb

extern "C" int pb_pair_products(int precision, int64_t n_vox, const void *X, const void *Y, const void *Z,
                                const void *U, const int32_t *pairs, int n_pairs, double s, void *out, void *stream) {
    if (n_vox < 1 || n_pairs < 0) return fail(PB_ERR_INVALID, "pb_pair_products: bad sizes");
    if (n_pairs == 0) return PB_OK;
    if (!X || !Y || !pairs || !out) return fail(PB_ERR_INVALID, "pb_pair_products: NULL argument");
    if ((Z == nullptr) != (U == nullptr)) return fail(PB_ERR_INVALID, "pb_pair_products: Z and U go together");
    size_t esz = precision == PB_F64 ? 8 : 4;
    if (precision != PB_F32 && precision != PB_F64) return fail(PB_ERR_INVALID, "bad precision");
    int threads = 256;
    int bx = grid_blocks(n_vox, threads, 2);
    for (int c0 = 0; c0 < n_pairs; c0 += PB_PAIR_MAX) {
        PairParams p;
        p.n = std::min(PB_PAIR_MAX, n_pairs - c0);
        for (int k = 0; k < p.n; ++k) {
            p.i[k] = pairs[2 * (c0 + k)];
            p.j[k] = pairs[2 * (c0 + k) + 1];
            if (p.i[k] < 0 || p.j[k] < 0) return fail(PB_ERR_INVALID, "pb_pair_products: negative map index");
        }
        dim3 grid(bx, p.n);
        void *o = (char *)out + (size_t)c0 * n_vox * esz;
        if (precision == PB_F32)
            pair_kernel<float><<<grid, threads, 0, as_stream(stream)>>>(n_vox, (const float *)X, (const float *)Y,
                                                                       (const float *)Z, (const float *)U, (float)s,
                                                                       (float *)o, p);
        else
            pair_kernel<double><<<grid, threads, 0, as_stream(stream)>>>(n_vox, (const double *)X, (const double *)Y,
                                                                        (const double *)Z, (const double *)U, s,
                                                                        (double *)o, p);
        PB_LAUNCH_CHECK("pb_pair_products");
    }
    return PB_OK;
}

extern "C" int pb_binned_filter(const pb_grid_t *g, int precision, const void *src, void *out, const double *edges,
                                int nk, const int32_t *ells, int n_ell, const double *coef, const void *w, int wpow,
                                double scale, void *stream) {
    Grid G;
    int st = make_grid(g, &G);
    if (st) return st;
    if (!src || !out || !edges || !ells || !coef) return fail(PB_ERR_INVALID, "pb_binned_filter: NULL argument");
    if (nk < 1 || nk > PB_RED_MAX_BINS) return fail(PB_ERR_INVALID, "pb_binned_filter: nk must be in [1, 64]");
    if (n_ell < 1 || n_ell > PB_RED_MAX_ELLS) return fail(PB_ERR_INVALID, "pb_binned_filter: n_ell must be in [1, 9]");
    if (wpow < -2 || wpow > 2) return fail(PB_ERR_INVALID, "pb_binned_filter: wpow must be in [-2, 2]");
    BinWParams p;
    for (int i = 0; i <= nk; ++i) {
        p.edges[i] = edges[i];
        if (i > 0 && !(edges[i] > edges[i - 1])) return fail(PB_ERR_INVALID, "pb_binned_filter: edges must increase");
    }
    for (int e = 0; e < n_ell; ++e) {
        if (ells[e] < 0 || ells[e] > 4) return fail(PB_ERR_INVALID, "pb_binned_filter: Legendre order must be in [0, 4]");
        p.ell[e] = (int8_t)ells[e];
    }
    p.nk = nk;
    p.n_ell = n_ell;
    p.wpow = w ? wpow : 0;
    p.scale = scale;
    int threads = 256;
    int blocks = grid_blocks(G.nhalf, threads);
    if (precision == PB_F32)
        binned_filter_kernel<float><<<blocks, threads, 0, as_stream(stream)>>>(G, (const float2 *)src, (float2 *)out,
                                                                               coef, (const float *)w, p);
    else if (precision == PB_F64)
        binned_filter_kernel<double><<<blocks, threads, 0, as_stream(stream)>>>(G, (const double2 *)src,
                                                                                (double2 *)out, coef, (const double *)w, p);
    else
        return fail(PB_ERR_INVALID, "bad precision");
    PB_LAUNCH_CHECK("pb_binned_filter");
    return PB_OK;
}
