// Band-limited map synthesis: the spectral filter followed by the inverse real 3D transform,
// computed as a pruned transform.
//
//   out[m](x) = sum_k F_m(k) e^{+2 pi i k.x / M}   (unnormalised, numpy irfftn x M^3 convention)
//   F_m(k)    = scale_m * src[src_m](k) * w(k)^wpow_m * Theta(lo_m <= |k| < hi_m) L_l1(mu) L_l2(mu)
//
// F_m vanishes outside the ball |k| < hi_m, so only the planes kz <= hi_m / kF_z, and in each
// plane only the columns and rows inside the band limit, carry data.  Three passes of
// batched 1D transforms (Stockham, mixed radix 2/3/4/5/8, in shared memory):
//   S1  per (map, kz plane, chunk of ky columns): gather + filter the source modes of each
//       column (kx inside the band), inverse transform along x -> U[m][kz][x][ky]
//   S2  per (map, kz plane, chunk of x rows): ky inside the band -> inverse transform along
//       y -> H[m][kz][x][y]
//   S3  per (map, x, chunk of y lines): the Hermitian half-line kz in [0, Kz] of two real
//       output lines packed into one complex transform along z -> out[m][x][y][z]
// U and H live in the caller's workspace.  The passes agree on which columns carry data
// through one device function (plane_radius), so S2 reads exactly what S1 wrote.
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>
#include <cuda_bf16.h>
#include "pb_common.cuh"

namespace pb {

constexpr int SY_MAX_MAPS = 64;
constexpr int SY_MAXF = 12;
constexpr int SY_THREADS = 512;
constexpr int SY_THREADS_Z = 768;  // 24 line groups: the radix-8 passes of 192 take one butterfly per thread
constexpr int SY_SMEM_BUDGET = 100 * 1024;

struct FftAxis {
    int n, np, lshift;  // length, number of radix passes, log2(lines per block)
    int rad[SY_MAXF];
};

struct SynthMap {
    double lo, hi, scale;
    int src, l1, l2, wpow;
    int kz_max;       // planes 0..kz_max
    int rx, ry;       // band half-widths in x and y (index units)
    int wu;           // U row width = 2 ry + 1
    int64_t u_off;    // complex offset of this map's U block
    int64_t h_off;    // complex offset of this map's H block
    int b1, b2, b3;   // first block of this map in S1, S2, S3
};

struct SynthParams {
    int n_maps;
    int n0, n1, n2, nh2;        // source grid
    int m0, m1, m2;             // output grid
    double kf0, kf1, kf2;
    int los;                    // line of sight of the Legendre weights (see Grid)
    double l0, l1, l2;
    int64_t src_stride;
    FftAxis ax, ay, az;
    int c1;                     // S1 column chunks per plane (max over maps)
    int tiled;                  // 0: out is [map][x][y][z]; 1: a tiled set (see tiled_c_byte)
    int t_maps, t_factor;       // the tiled set's map and factor-map counts
    SynthMap maps[SY_MAX_MAPS];
};

// ---- complex helpers ----------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cmuli(float2 a) { return make_float2(-a.y, a.x); }  // i * a
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cmuli(double2 a) { return make_double2(-a.y, a.x); }

template <typename T> __device__ __forceinline__ typename cplx<T>::type cmake(double x, double y);
template <> __device__ __forceinline__ float2 cmake<float>(double x, double y) { return make_float2((float)x, (float)y); }
template <> __device__ __forceinline__ double2 cmake<double>(double x, double y) { return make_double2(x, y); }

// ---- small inverse DFTs (sign +) in registers -----------------------------------------
template <typename T, typename C>
__device__ __forceinline__ void idft2(C &a, C &b) {
    C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <typename T, typename C>
__device__ __forceinline__ void idft3(C *v) {
    const T h = (T)0.86602540378443864676;  // sqrt(3) / 2
    C s = cadd(v[1], v[2]);
    C d = cscale(cmuli(csub(v[1], v[2])), h);
    C t = csub(v[0], cscale(s, (T)0.5));
    v[0] = cadd(v[0], s);
    v[1] = cadd(t, d);
    v[2] = csub(t, d);
}

template <typename T, typename C>
__device__ __forceinline__ void idft4(C &v0, C &v1, C &v2, C &v3) {
    C t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = cmuli(csub(v1, v3));
    v0 = cadd(t0, t2);
    v2 = csub(t0, t2);
    v1 = cadd(t1, t3);
    v3 = csub(t1, t3);
}

template <typename T, typename C>
__device__ __forceinline__ void idft5(C *v) {
    const T c1 = (T)0.30901699437494742410, c2 = (T)-0.80901699437494742410;
    const T s1 = (T)0.95105651629515357212, s2 = (T)0.58778525229247312917;
    C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    C x0 = v[0];
    C r1 = cadd(x0, cadd(cscale(a1, c1), cscale(a2, c2)));
    C r2 = cadd(x0, cadd(cscale(a1, c2), cscale(a2, c1)));
    C i1 = cmuli(cadd(cscale(b1, s1), cscale(b2, s2)));
    C i2 = cmuli(csub(cscale(b1, s2), cscale(b2, s1)));
    v[0] = cadd(x0, cadd(a1, a2));
    v[1] = cadd(r1, i1);
    v[4] = csub(r1, i1);
    v[2] = cadd(r2, i2);
    v[3] = csub(r2, i2);
}

template <typename T, typename C>
__device__ __forceinline__ void idft8(C *v) {
    const T r = (T)0.70710678118654752440;
    // even / odd halves
    idft4<T, C>(v[0], v[2], v[4], v[6]);
    idft4<T, C>(v[1], v[3], v[5], v[7]);
    // twiddles e^{+i pi k / 4} on the odd half
    C o1 = cscale(cadd(v[3], cmuli(v[3])), r);           // (1 + i)/sqrt2
    C o2 = cmuli(v[5]);                                   // i
    C o3 = cscale(csub(cmuli(v[7]), v[7]), r);            // (-1 + i)/sqrt2
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1);
    v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2);
    v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3);
    v[7] = csub(e3, o3);
}

// One Stockham pass of radix R over `lines` lines stored at stride ld in `src`, written to
// `dst` (same layout); Ns = product of the radices of the previous passes; tw[t] =
// e^{+2 pi i t / n}.  Threads run line-fastest: thread t takes line t mod L (L = 2^lshift
// lines per block) and butterflies j = t / L, t / L + NG, ... (NG = blockDim / L), so a
// warp touches 32 different lines at the same position and the line stride ld = n + 1
// keeps those accesses on distinct banks.  j / Ns and j mod Ns are carried incrementally.
template <int R, typename T>
__device__ __forceinline__ void stockham_pass(const typename cplx<T>::type *src, typename cplx<T>::type *dst,
                                              int ld, int lines, int lshift, int n, int Ns,
                                              const typename cplx<T>::type *tw) {
    using C = typename cplx<T>::type;
    const int nb = n / R;
    const int line = threadIdx.x & ((1 << lshift) - 1);
    const int NG = blockDim.x >> lshift;
    if (line >= lines) return;
    const int tstep = n / (Ns * R);
    int j = threadIdx.x >> lshift;
    int jq = j / Ns, jm = j - jq * Ns;
    const int sq = NG / Ns, sm = NG - sq * Ns;
    const C *s = src + (int64_t)line * ld;
    C *d = dst + (int64_t)line * ld;
    for (; j < nb; j += NG) {
        C v[R];
        v[0] = s[j];
#pragma unroll
        for (int r = 1; r < R; ++r) {
            C x = s[j + r * nb];
            if (jm > 0) x = cmul(x, tw[r * jm * tstep]);
            v[r] = x;
        }
        if (R == 2) idft2<T, C>(v[0], v[1]);
        else if (R == 3) idft3<T, C>(v);
        else if (R == 4) idft4<T, C>(v[0], v[1], v[2], v[3]);
        else if (R == 5) idft5<T, C>(v);
        else idft8<T, C>(v);
        const int o = jq * Ns * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) d[o + r * Ns] = v[r];
        jq += sq;
        jm += sm;
        if (jm >= Ns) {
            jm -= Ns;
            ++jq;
        }
    }
}

// Radix plan of a length: 8s first, then 4, 2, 3, 5 (so Ns stays a power of two through the
// radix-2^k passes).  Shared by the compile-time and the run-time forms.
__host__ __device__ constexpr int radix_of(int n) {
    return n % 8 == 0 ? 8 : n % 4 == 0 ? 4 : n % 2 == 0 ? 2 : n % 3 == 0 ? 3 : n % 5 == 0 ? 5 : 0;
}
__host__ __device__ constexpr int radix_at(int n, int q) {
    for (int i = 0; i < q; ++i) n /= radix_of(n);
    return radix_of(n);
}
__host__ __device__ constexpr int pass_count(int n) {
    int c = 0;
    while (n > 1) {
        const int f = radix_of(n);
        if (f == 0) return -1;
        n /= f;
        ++c;
    }
    return c;
}

// Compile-time-length pass: nb, Ns, the twiddle stride and the line stride are constants,
// so the index arithmetic folds away.
template <int R, typename T, int N, int NS>
__device__ __forceinline__ void stockham_pass_ct(const typename cplx<T>::type *src, typename cplx<T>::type *dst,
                                                 int lines, int lshift, const typename cplx<T>::type *tw) {
    using C = typename cplx<T>::type;
    constexpr int nb = N / R;
    constexpr int tstep = N / (NS * R);
    constexpr int ld = N + 1;
    const int line = threadIdx.x & ((1 << lshift) - 1);
    const int NG = blockDim.x >> lshift;
    if (line >= lines) return;
    const C *s = src + line * ld;
    C *d = dst + line * ld;
    for (int j = threadIdx.x >> lshift; j < nb; j += NG) {
        const int jm = j % NS, jq = j / NS;
        C v[R];
        v[0] = s[j];
#pragma unroll
        for (int r = 1; r < R; ++r) {
            C x = s[j + r * nb];
            if (NS > 1) x = cmul(x, tw[r * jm * tstep]);
            v[r] = x;
        }
        if (R == 2) idft2<T, C>(v[0], v[1]);
        else if (R == 3) idft3<T, C>(v);
        else if (R == 4) idft4<T, C>(v[0], v[1], v[2], v[3]);
        else if (R == 5) idft5<T, C>(v);
        else idft8<T, C>(v);
        const int o = jq * (NS * R) + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) d[o + r * NS] = v[r];
    }
}

template <typename T, int N, int Q, int NS>
__device__ __forceinline__ void passes_ct(typename cplx<T>::type *&src, typename cplx<T>::type *&dst, int lines,
                                          int lshift, const typename cplx<T>::type *tw) {
    if constexpr (Q < pass_count(N)) {
        constexpr int R = radix_at(N, Q);
        stockham_pass_ct<R, T, N, NS>(src, dst, lines, lshift, tw);
        __syncthreads();
        typename cplx<T>::type *t = src;
        src = dst;
        dst = t;
        passes_ct<T, N, Q + 1, NS * R>(src, dst, lines, lshift, tw);
    }
}

__host__ __device__ constexpr int ns_at(int n, int q) {
    int ns = 1;
    for (int i = 0; i < q; ++i) ns *= radix_at(n, i);
    return ns;
}

// A compile-time pass whose operands come from and go to functors: v[r] = ldf(line, j + r nb)
// (twiddled), stf(line, o + r Ns, v[r]).  ELEM: threads run j-fastest along a line (for
// loads or stores that are contiguous along the line in global memory); otherwise
// line-fastest as in stockham_pass_ct.
template <int R, typename T, int N, int NS, bool ELEM, typename LD, typename ST>
__device__ __forceinline__ void io_pass(int lines, int lshift, const typename cplx<T>::type *tw, LD &&ldf,
                                        ST &&stf) {
    using C = typename cplx<T>::type;
    constexpr int nb = N / R;
    constexpr int tstep = N / (NS * R);
    auto body = [&](int line, int j) {
        const int jm = j % NS, jq = j / NS;
        C v[R];
        v[0] = ldf(line, j);
#pragma unroll
        for (int r = 1; r < R; ++r) {
            C x = ldf(line, j + r * nb);
            if (NS > 1) x = cmul(x, tw[r * jm * tstep]);
            v[r] = x;
        }
        if (R == 2) idft2<T, C>(v[0], v[1]);
        else if (R == 3) idft3<T, C>(v);
        else if (R == 4) idft4<T, C>(v[0], v[1], v[2], v[3]);
        else if (R == 5) idft5<T, C>(v);
        else idft8<T, C>(v);
        const int o = jq * (NS * R) + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) stf(line, o + r * NS, v[r]);
    };
    if (ELEM) {
        for (int it = threadIdx.x; it < lines * nb; it += blockDim.x) {
            const int line = it / nb;
            body(line, it - line * nb);
        }
    } else {
        const int line = threadIdx.x & ((1 << lshift) - 1);
        if (line >= lines) return;
        for (int j = threadIdx.x >> lshift; j < nb; j += blockDim.x >> lshift) body(line, j);
    }
}

template <typename T, int N, int Q, int QEND>
__device__ __forceinline__ void smem_passes(typename cplx<T>::type *&src, typename cplx<T>::type *&dst, int lines,
                                            int lshift, const typename cplx<T>::type *tw) {
    if constexpr (Q < QEND) {
        stockham_pass_ct<radix_at(N, Q), T, N, ns_at(N, Q)>(src, dst, lines, lshift, tw);
        __syncthreads();
        typename cplx<T>::type *t = src;
        src = dst;
        dst = t;
        smem_passes<T, N, Q + 1, QEND>(src, dst, lines, lshift, tw);
    }
}

// Compile-time length, data in b0 (line stride N + 1): every pass but the last in shared
// memory, the last one straight to stf(line, element, value).
template <typename T, int N, bool LAST_ELEM, typename ST>
__device__ __forceinline__ void line_ifft_tail(typename cplx<T>::type *b0, typename cplx<T>::type *b1, int lines,
                                               int lshift, const typename cplx<T>::type *tw, ST &&stf) {
    using C = typename cplx<T>::type;
    constexpr int P = pass_count(N);
    C *src = b0, *dst = b1;
    smem_passes<T, N, 0, P - 1>(src, dst, lines, lshift, tw);
    const C *s = src;
    io_pass<radix_at(N, P - 1), T, N, ns_at(N, P - 1), LAST_ELEM>(
        lines, lshift, tw, [&](int line, int e) { return s[line * (N + 1) + e]; }, stf);
}

// Compile-time length, first pass straight from ldf(line, element) (line-fastest), last pass
// straight to stf; needs at least two passes.
template <typename T, int N, bool LAST_ELEM, typename LD, typename ST>
__device__ __forceinline__ void line_ifft_io(typename cplx<T>::type *b0, typename cplx<T>::type *b1, int lines,
                                             int lshift, const typename cplx<T>::type *tw, LD &&ldf, ST &&stf) {
    using C = typename cplx<T>::type;
    constexpr int P = pass_count(N);
    static_assert(P >= 2, "line_ifft_io needs two passes");
    io_pass<radix_at(N, 0), T, N, 1, false>(lines, lshift, tw, ldf,
                                            [&](int line, int e, C v) { b0[line * (N + 1) + e] = v; });
    __syncthreads();
    C *src = b0, *dst = b1;
    smem_passes<T, N, 1, P - 1>(src, dst, lines, lshift, tw);
    const C *s = src;
    io_pass<radix_at(N, P - 1), T, N, ns_at(N, P - 1), LAST_ELEM>(
        lines, lshift, tw, [&](int line, int e) { return s[line * (N + 1) + e]; }, stf);
}

// All passes of one axis; data starts in b0, returns the buffer holding the result.
// N > 0: compile-time length; N == 0: the length and radices of `ax` at run time.
template <typename T, int N>
__device__ typename cplx<T>::type *line_ifft(typename cplx<T>::type *b0, typename cplx<T>::type *b1, int ld,
                                             int lines, const FftAxis &ax, const typename cplx<T>::type *tw) {
    using C = typename cplx<T>::type;
    C *src = b0, *dst = b1;
    if constexpr (N > 0) {
        passes_ct<T, N, 0, 1>(src, dst, lines, ax.lshift, tw);
        return src;
    }
    int Ns = 1;
    for (int q = 0; q < ax.np; ++q) {
        const int R = ax.rad[q];
        switch (R) {
            case 2: stockham_pass<2, T>(src, dst, ld, lines, ax.lshift, ax.n, Ns, tw); break;
            case 3: stockham_pass<3, T>(src, dst, ld, lines, ax.lshift, ax.n, Ns, tw); break;
            case 4: stockham_pass<4, T>(src, dst, ld, lines, ax.lshift, ax.n, Ns, tw); break;
            case 5: stockham_pass<5, T>(src, dst, ld, lines, ax.lshift, ax.n, Ns, tw); break;
            default: stockham_pass<8, T>(src, dst, ld, lines, ax.lshift, ax.n, Ns, tw); break;
        }
        __syncthreads();
        Ns *= R;
        C *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

template <typename T>
__device__ __forceinline__ void make_twiddles(typename cplx<T>::type *tw, int n) {
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        if (sizeof(T) == 4) {
            // 2t/n is exact in FP32 for n <= 2^23
            float sf, cf;
            sincospif(2.0f * (float)t / (float)n, &sf, &cf);
            tw[t] = cmake<T>(cf, sf);
        } else {
            double sd, cd;
            sincospi(2.0 * (double)t / (double)n, &sd, &cd);
            tw[t] = cmake<T>(cd, sd);
        }
    }
}

// |ky| bound of plane kz for a map of upper edge hi (one extra column of margin; the exact
// membership test happens per mode).  -1: the plane is empty.
__device__ __forceinline__ int plane_radius(const SynthParams &p, const SynthMap &mp, int kz) {
    const double kzv = (double)kz * p.kf2;
    const double r2 = mp.hi * mp.hi - kzv * kzv;
    if (r2 < 0.0) return -1;
    int r = (int)floor(sqrt(r2) / p.kf1) + 1;
    return r < mp.ry ? r : mp.ry;
}

__device__ __forceinline__ int find_map(const SynthParams &p, int b, int which) {
    int m = 0;
    for (int i = 1; i < p.n_maps; ++i) {
        const int first = which == 1 ? p.maps[i].b1 : (which == 2 ? p.maps[i].b2 : p.maps[i].b3);
        if (b >= first) m = i;
    }
    return m;
}

// ---- S1: gather + filter + transform along x ------------------------------------------
// S: the source spectrum's element type, the maps' complex type or (FP32 maps) complex FP64:
// the filter product is formed in FP64 and rounded to T once
template <typename T, int N, typename S = typename cplx<T>::type>
__global__ void __launch_bounds__(SY_THREADS) synth_x_kernel(SynthParams p, const S *src, const T *w,
                                                             typename cplx<T>::type *U) {
    using C = typename cplx<T>::type;
    extern __shared__ __align__(16) unsigned char sy_smem[];
    const FftAxis &ax = p.ax;
    const int n = N > 0 ? N : ax.n, ld = n + 1, L = 1 << ax.lshift;
    C *tw = reinterpret_cast<C *>(sy_smem);
    C *b0 = tw + n;
    C *b1 = b0 + L * ld;
    const int m = find_map(p, blockIdx.x, 1);
    const SynthMap mp = p.maps[m];
    const int local = blockIdx.x - mp.b1;
    const int kz = local / p.c1;
    const int chunk = local - kz * p.c1;
    const int R = plane_radius(p, mp, kz);
    const int c0 = chunk * L;  // first column index (ky = c - ry)
    const int col_first = max(c0, mp.ry - R), col_last = min(c0 + L - 1, mp.ry + R);
    if (R < 0 || col_first > col_last) return;
    const int lines = col_last - c0 + 1;  // lines below col_first stay 0
    make_twiddles<T>(tw, n);
    const S *s = src ? src + (int64_t)mp.src * p.src_stride : nullptr;  // NULL: unit spectrum
    const double kzz = __dmul_rn((double)kz, p.kf2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int line = warp; line < lines; line += nw) {
        const int c = c0 + line;
        const int ky = c - mp.ry;
        const double kyv = __dmul_rn((double)ky, p.kf1);
        const int sj = ky < 0 ? ky + p.n1 : ky;
        C *row = b0 + (int64_t)line * ld;
        for (int e = lane; e < n; e += 32) {
            const int kx = e < (n >> 1) ? e : e - n;
            C v = cmake<T>(0.0, 0.0);
            if (c >= col_first && kx >= -mp.rx && kx <= mp.rx) {
                const double kxv = __dmul_rn((double)kx, p.kf0);
                const double kk = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(kxv, kxv), __dmul_rn(kyv, kyv)),
                                                       __dmul_rn(kzz, kzz)));
                if (mp.lo <= kk && kk < mp.hi) {
                    const double mu =
                        kk != 0.0 ? __ddiv_rn(k_dot_los(p.los, p.l0, p.l1, p.l2, kxv, kyv, kzz), kk) : 0.0;
                    const int si = kx < 0 ? kx + p.n0 : kx;
                    const int64_t sidx = ((int64_t)si * p.n1 + sj) * p.nh2 + kz;
                    double f = mp.scale * legendre(mp.l1, mu) * legendre(mp.l2, mu);
                    if (mp.wpow != 0) {
                        const double wv = (double)w[sidx];
                        if (mp.wpow == 1) f *= wv;
                        else if (mp.wpow == 2) f *= wv * wv;
                        else f = wv != 0.0 ? f / wv : 0.0;
                    }
                    if (s) {
                        const S x = s[sidx];
                        v = cmake<T>((double)x.x * f, (double)x.y * f);
                    } else {
                        v = cmake<T>(f, 0.0);
                    }
                }
            }
            row[e] = v;
        }
    }
    __syncthreads();
    // U[m][kz][x][c]: consecutive threads take consecutive columns
    C *u = U + mp.u_off + (int64_t)kz * n * mp.wu;
    if constexpr (N > 0) {
        line_ifft_tail<T, N, false>(b0, b1, lines, ax.lshift, tw, [&](int line, int x, C v) {
            const int c = c0 + line;
            if (c >= col_first) u[(int64_t)x * mp.wu + c] = v;
        });
    } else {
        C *res = line_ifft<T, N>(b0, b1, ld, lines, ax, tw);
        const int line = threadIdx.x & (L - 1), NG = blockDim.x >> ax.lshift;
        const int c = c0 + line;
        if (line < lines && c >= col_first)
            for (int x = threadIdx.x >> ax.lshift; x < n; x += NG)
                u[(int64_t)x * mp.wu + c] = res[(int64_t)line * ld + x];
    }
}

// ---- S2: transform along y --------------------------------------------------------------
template <typename T, int N>
__global__ void __launch_bounds__(SY_THREADS) synth_y_kernel(SynthParams p, const typename cplx<T>::type *U,
                                                             typename cplx<T>::type *H) {
    using C = typename cplx<T>::type;
    extern __shared__ __align__(16) unsigned char sy_smem[];
    const FftAxis &ay = p.ay;
    const int n = N > 0 ? N : ay.n, ld = n + 1, L = 1 << ay.lshift;
    C *tw = reinterpret_cast<C *>(sy_smem);
    C *b0 = tw + n;
    C *b1 = b0 + L * ld;
    const int m = find_map(p, blockIdx.x, 2);
    const SynthMap mp = p.maps[m];
    const int local = blockIdx.x - mp.b2;
    const int xchunks = (p.m0 + L - 1) >> ay.lshift;
    const int kz = local / xchunks;
    const int x0 = (local - kz * xchunks) * L;
    const int lines = min(L, p.m0 - x0);
    const int R = plane_radius(p, mp, kz);
    make_twiddles<T>(tw, n);
    const C *u = U + mp.u_off + (int64_t)kz * p.m0 * mp.wu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    // loads of a batch are issued before any of them is stored, so each thread keeps
    // several global reads in flight
    constexpr int UB = 8;
    for (int line = warp; line < lines; line += nw) {
        const C *urow = u + (int64_t)(x0 + line) * mp.wu + mp.ry;
        C *row = b0 + (int64_t)line * ld;
        for (int e0 = lane; e0 < n; e0 += 32 * UB) {
            C v[UB];
#pragma unroll
            for (int q = 0; q < UB; ++q) {
                const int e = e0 + 32 * q;
                const int ky = e < (n >> 1) ? e : e - n;
                v[q] = (e < n && ky >= -R && ky <= R) ? urow[ky] : cmake<T>(0.0, 0.0);
            }
#pragma unroll
            for (int q = 0; q < UB; ++q)
                if (e0 + 32 * q < n) row[e0 + 32 * q] = v[q];
        }
    }
    __syncthreads();
    C *h = H + mp.h_off + ((int64_t)kz * p.m0 + x0) * p.m1;
    if constexpr (N > 0) {
        line_ifft_tail<T, N, true>(b0, b1, lines, ay.lshift, tw,
                                   [&](int line, int y, C v) { h[(int64_t)line * p.m1 + y] = v; });
    } else {
        C *res = line_ifft<T, N>(b0, b1, ld, lines, ay, tw);
        for (int line = warp; line < lines; line += nw) {
            const C *row = res + (int64_t)line * ld;
            C *hrow = h + (int64_t)line * p.m1;
            for (int y = lane; y < n; y += 32) hrow[y] = row[y];
        }
    }
}

// ---- tiled-set output ------------------------------------------------------------------
// voxel v of map m into a tiled set: FP32 copy of a factor map, bf16 hi and lo parts
__device__ __forceinline__ void tiled_put(const SynthParams &p, int m, int64_t v, float val, char *out) {
    if (m < p.t_factor) *reinterpret_cast<float *>(out + tiled_factor_byte(v, m, p.t_maps, p.t_factor)) = val;
    const __nv_bfloat16 hi = __float2bfloat16_rn(val);
    const __nv_bfloat16 lo = __float2bfloat16_rn(val - __bfloat162float(hi));
    *reinterpret_cast<__nv_bfloat16 *>(out + tiled_c_byte(v, m, p.t_maps, p.t_factor)) = hi;
    *reinterpret_cast<__nv_bfloat16 *>(out + tiled_c_byte(v, tiled_cpad(p.t_maps) + m, p.t_maps, p.t_factor)) = lo;
}

// Staged values of map m (rows of NN voxels, row stride lds in stg; voxels v0 .. v0 + rows NN
// - 1) into a tiled set, by warps wk = 0 .. nw - 1 of a group (the caller's warp index in it).
// Each warp takes 64 consecutive voxels per step, a lane two neighbours: two 128-byte rows of
// factor slabs (8-byte stores) and four 32-byte K-step rows each of the hi and lo parts
// (bf16x2 stores), so the stores fill whole sectors; offsets inside a tile are per lane and
// computed once per map, the tile base per chunk.  Per voxel (tiled_put) when the run is not
// 64-aligned.
template <int NN>
__device__ void flush_tiled(const SynthParams &p, int m, int64_t v0, int rows, int lds, const float *stg, char *out,
                            int wk, int nw) {
    const int count = rows * NN;
    const int lane = threadIdx.x & 31;
    if ((NN & 1) != 0 || (v0 & 63) != 0 || (count & 63) != 0) {
        for (int i = wk * 32 + lane; i < count; i += nw * 32) {
            const int r = i / NN, z = i - r * NN;
            tiled_put(p, m, v0 + i, stg[r * lds + z], out);
        }
        return;
    }
    const int F = tiled_frows(p.t_factor), P = tiled_cpad(p.t_maps);
    const int64_t tb = tiled_tile_bytes(p.t_maps, p.t_factor);
    const bool factor = m < p.t_factor;
    // lane j holds voxels 2j, 2j + 1 of the chunk: slab j / 16, 4-voxel chunk (j % 16) / 2 of
    // it; K step j / 8, 8-voxel half (j / 4) % 2, element 2 (j % 4)
    const uint32_t off_f = (uint32_t)(lane >> 4) * F * 128u + (uint32_t)m * 128u +
                           ((((uint32_t)(lane & 15) >> 1) ^ ((uint32_t)m & 7u)) << 4) + (lane & 1) * 8;
    auto c_off = [&](int r) {
        return (uint32_t)((lane >> 3) * 64 * P + (r >> 3) * 256 + (r & 7) * 32 +
                          ((((lane >> 2) & 1) ^ ((r >> 2) & 1)) << 4) + (lane & 3) * 4);
    };
    const uint32_t off_hi = c_off(m), off_lo = c_off(P + m);
    for (int u = wk * 64; u < count; u += nw * 64) {
        const int i = u + 2 * lane, r = i / NN, z = i - r * NN;  // NN even: both voxels in row r
        const float x0 = stg[r * lds + z], x1 = stg[r * lds + z + 1];
        const int64_t v = v0 + u;  // 64-aligned: two slabs, four K steps of one tile
        const int w = (int)(v & (TILED_VOX - 1));
        char *const tile = out + (v >> 7) * tb;
        if (factor) *reinterpret_cast<float2 *>(tile + (w >> 5) * F * 128 + off_f) = make_float2(x0, x1);
        const __nv_bfloat162 hb = __floats2bfloat162_rn(x0, x1);
        const __nv_bfloat162 lb = __floats2bfloat162_rn(x0 - __low2float(hb), x1 - __high2float(hb));
        char *const cop = tile + 512 * F + (w >> 4) * 64 * P;
        *reinterpret_cast<__nv_bfloat162 *>(cop + off_hi) = hb;
        *reinterpret_cast<__nv_bfloat162 *>(cop + off_lo) = lb;
    }
}

// ---- S3: real transform along z, two output lines per complex transform -----------------
template <typename T, int N>
// (FP32: two 768-thread blocks resident per SM, 42 registers; FP64 keeps its registers)
__global__ void __launch_bounds__(SY_THREADS_Z, sizeof(T) == 4 ? 2 : 1) synth_z_kernel(SynthParams p, const typename cplx<T>::type *H,
                                                             T *out) {
    using C = typename cplx<T>::type;
    extern __shared__ __align__(16) unsigned char sy_smem[];
    const FftAxis &az = p.az;
    const int n = N > 0 ? N : az.n, ld = n + 1, L = 1 << az.lshift;
    C *tw = reinterpret_cast<C *>(sy_smem);
    C *b0 = tw + n;
    C *b1 = b0 + L * ld;
    const int m = find_map(p, blockIdx.x, 3);
    const SynthMap mp = p.maps[m];
    const int local = blockIdx.x - mp.b3;
    const int ychunks = (p.m1 + 2 * L - 1) / (2 * L);
    const int x = local / ychunks;
    const int y0 = (local - x * ychunks) * 2 * L;
    const int ny = min(2 * L, p.m1 - y0);
    const int lines = (ny + 1) >> 1;
    const int K = mp.kz_max;
    make_twiddles<T>(tw, n);  // made visible by the barrier after the first pass
    const int64_t plane = (int64_t)p.m0 * p.m1;
    // voxel v0 + yy m2 + z of map m: plain [map][voxel] rows, or the slab layout of a tiled set
    const int64_t v0 = ((int64_t)x * p.m1 + y0) * p.m2;
    T *const o = out + (int64_t)m * plane * p.m2 + v0;
    const int tiled = p.tiled;
    auto put = [&](int yy, int z, T val) {
        if (!tiled) o[(int64_t)yy * p.m2 + z] = val;
        else tiled_put(p, m, v0 + (int64_t)yy * p.m2 + z, (float)val, reinterpret_cast<char *>(out));
    };
    if constexpr (N > 0 && pass_count(N) >= 2) {
        // a tiled set's rows (2 L lines of n values) are staged in the transform buffer the last
        // pass does not read (b1 after an even number of shared-memory passes, else b0) and
        // written out together
        float *const stg = reinterpret_cast<float *>((pass_count(N) - 2) % 2 == 0 ? b1 : b0);
        constexpr int LDS = N + 1;  // odd row stride: the last pass's lanes write different rows
        // first pass straight from H (a warp reads the (y, y+1) pairs of 32 lines at one kz:
        // 512 contiguous bytes; it needs no twiddles), last pass straight to the real rows
        const C *hb = H + mp.h_off + (int64_t)x * p.m1 + y0;
        line_ifft_io<T, N, true>(
            b0, b1, lines, az.lshift, tw,
            [&](int line, int e) -> C {
                int kz;
                bool mirror = false;
                if (e <= K) {
                    kz = e;
                } else if (e >= N - K) {
                    kz = N - e;
                    mirror = true;
                } else {
                    return cmake<T>(0.0, 0.0);
                }
                const C *hl = hb + 2 * line + kz * plane;
                C a, b;
                if constexpr (std::is_same<T, float>::value) {
                    const float4 q = *reinterpret_cast<const float4 *>(hl);
                    a = make_float2(q.x, q.y);
                    b = make_float2(q.z, q.w);
                } else {
                    a = hl[0];
                    b = hl[1];
                }
                if (kz == 0) return cmake<T>((double)a.x, (double)b.x);
                C r;
                if (!mirror) {
                    r.x = a.x - b.y;
                    r.y = a.y + b.x;
                } else {
                    r.x = a.x + b.y;
                    r.y = b.x - a.y;
                }
                return r;
            },
            [&](int line, int z, C v) {
                if (tiled) {
                    stg[(2 * line) * LDS + z] = (float)v.x;
                    stg[(2 * line + 1) * LDS + z] = (float)v.y;
                } else {
                    put(2 * line, z, v.x);
                    put(2 * line + 1, z, v.y);
                }
            });
        if (tiled) {
            __syncthreads();
            flush_tiled<N>(p, m, v0, ny, LDS, stg, reinterpret_cast<char *>(out), threadIdx.x >> 5, blockDim.x >> 5);
        }
        return;
    }
    // line-fastest: consecutive threads read consecutive (y, y+1) pairs of one kz row
    const int line = threadIdx.x & (L - 1), NG = blockDim.x >> az.lshift;
    if (line < lines) {
        C *d = b0 + (int64_t)line * ld;
        for (int e = (threadIdx.x >> az.lshift) + K + 1; e < n - K; e += NG) d[e] = cmake<T>(0.0, 0.0);
        const C *h = H + mp.h_off + (int64_t)x * p.m1 + y0 + 2 * line;
        const bool has_b = 2 * line + 1 < ny;
        constexpr int UB = 4;  // loads in flight per thread
        for (int kz0 = threadIdx.x >> az.lshift; kz0 <= K; kz0 += UB * NG) {
            C a[UB], b[UB];
#pragma unroll
            for (int q = 0; q < UB; ++q) {
                const int kz = kz0 + q * NG;
                a[q] = kz <= K ? h[kz * plane] : cmake<T>(0.0, 0.0);
                b[q] = (kz <= K && has_b) ? h[kz * plane + 1] : cmake<T>(0.0, 0.0);
            }
#pragma unroll
            for (int q = 0; q < UB; ++q) {
                const int kz = kz0 + q * NG;
                if (kz > K) break;
                if (kz == 0) {
                    d[0] = cmake<T>((double)a[q].x, (double)b[q].x);
                } else {
                    C dp, dm;
                    dp.x = a[q].x - b[q].y;
                    dp.y = a[q].y + b[q].x;
                    dm.x = a[q].x + b[q].y;
                    dm.y = b[q].x - a[q].y;
                    d[kz] = dp;
                    d[n - kz] = dm;
                }
            }
        }
    }
    __syncthreads();
    C *res = line_ifft<T, N>(b0, b1, ld, lines, az, tw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int yy = warp; yy < ny; yy += nw) {
        const C *row = res + (int64_t)(yy >> 1) * ld;
        if (yy & 1)
            for (int z = lane; z < n; z += 32) put(yy, z, row[z].y);
        else
            for (int z = lane; z < n; z += 32) put(yy, z, row[z].x);
    }
}

// ---- S3 for a tiled set: a block per (x, 2 LY y-lines, group of SY_TMAPS maps) --------------
// Its L = SY_TMAPS LY complex lines are (map, y pair) combinations (line l: map g0 SY_TMAPS +
// l / LY, y pair l % LY), so the block writes neighbouring maps' rows of the same tiles -- one
// 8-row atom of each factor slab and K step -- together instead of one map's row in many tiles.
constexpr int SY_TMAPS = 8;  // a power of two (line -> map by shift)

template <int N>
__global__ void __launch_bounds__(SY_THREADS_Z, 2) synth_z_tiled_kernel(SynthParams p, const float2 *H, char *out) {
    extern __shared__ __align__(16) unsigned char sy_smem[];
    const FftAxis &az = p.az;
    const int L = 1 << az.lshift, LY = L / SY_TMAPS, ly_shift = az.lshift - 3;  // SY_TMAPS = 8
    float2 *tw = reinterpret_cast<float2 *>(sy_smem);
    float2 *b0 = tw + N;
    float2 *b1 = b0 + L * (N + 1);
    const int ychunks = (p.m1 + 2 * LY - 1) / (2 * LY), mgroups = (p.n_maps + SY_TMAPS - 1) / SY_TMAPS;
    int b = blockIdx.x;
    const int g0 = b % mgroups;
    b /= mgroups;
    const int yc = b % ychunks, x = b / ychunks;
    const int y0 = yc * 2 * LY, ny = min(2 * LY, p.m1 - y0);
    const int nm = min(SY_TMAPS, p.n_maps - SY_TMAPS * g0);
    make_twiddles<float>(tw, N);  // made visible by the barrier after the first pass
    const int64_t plane = (int64_t)p.m0 * p.m1;
    float *const stg = reinterpret_cast<float *>((pass_count(N) - 2) % 2 == 0 ? b1 : b0);
    constexpr int LDS = N + 1;
    line_ifft_io<float, N, true>(
        b0, b1, nm * LY, az.lshift, tw,
        [&](int line, int e) -> float2 {
            const int mi = line >> ly_shift, y = y0 + 2 * (line & (LY - 1));
            const SynthMap &mp = p.maps[SY_TMAPS * g0 + mi];
            const int K = mp.kz_max;
            int kz;
            bool mirror = false;
            if (y >= p.m1) return make_float2(0.f, 0.f);
            if (e <= K) {
                kz = e;
            } else if (e >= N - K) {
                kz = N - e;
                mirror = true;
            } else {
                return make_float2(0.f, 0.f);
            }
            // the (y, y + 1) pair of line: one 16-byte load (m1 even)
            const float4 q = *reinterpret_cast<const float4 *>(H + mp.h_off + kz * plane + (int64_t)x * p.m1 + y);
            const float2 a = make_float2(q.x, q.y), c = make_float2(q.z, q.w);
            if (kz == 0) return make_float2(a.x, c.x);
            return mirror ? make_float2(a.x + c.y, c.x - a.y) : make_float2(a.x - c.y, a.y + c.x);
        },
        [&](int line, int z, float2 v) {
            stg[(2 * line) * LDS + z] = v.x;
            stg[(2 * line + 1) * LDS + z] = v.y;
        });
    __syncthreads();
    const int64_t v0 = ((int64_t)x * p.m1 + y0) * p.m2;
    // a group of warps per map, so each warp sets up one map's offsets and stores many chunks
    const int nwb = blockDim.x >> 5, wpm = max(1, nwb / nm), warp = threadIdx.x >> 5;
    for (int mi = warp / wpm; mi < nm; mi += max(1, nwb / wpm))
        flush_tiled<N>(p, SY_TMAPS * g0 + mi, v0, ny, LDS, stg + 2 * mi * LY * LDS, out, warp % wpm, wpm);
}

// ---- host side ----------------------------------------------------------------------------
static bool factor_axis(int n, FftAxis &ax) {
    ax.n = n;
    ax.np = 0;
    int r = n;
    while (r > 1 && ax.np < SY_MAXF) {
        int f = 0;
        if (r % 8 == 0) f = 8;
        else if (r % 4 == 0) f = 4;
        else if (r % 2 == 0) f = 2;
        else if (r % 3 == 0) f = 3;
        else if (r % 5 == 0) f = 5;
        else return false;
        ax.rad[ax.np++] = f;
        r /= f;
    }
    return r == 1;
}

template <typename C>
static int lines_for(int n, int cap) {
    int L = 32;
    while (L > 1 && (int64_t)(2 * L * (n + 1) + n) * (int64_t)sizeof(C) > SY_SMEM_BUDGET) L >>= 1;
    return std::min(L, cap);
}

struct SynthLayout {
    SynthParams p;
    int64_t u_elems, h_elems;
    int nb1, nb2, nb3;
};

static int synth_layout(const pb_grid_t *g, const int32_t *out_n, int precision, int n_maps, const double *lo,
                        const double *hi, const int32_t *src_idx, const int32_t *l1, const int32_t *l2,
                        const double *scale, const int32_t *wpow, int64_t src_stride, SynthLayout *L) {
    Grid G;
    int st = make_grid(g, &G);
    if (st) return st;
    if (!out_n) return fail(PB_ERR_INVALID, "pb_shell_synth: out_n is NULL");
    if (n_maps < 1 || n_maps > SY_MAX_MAPS) return fail(PB_ERR_INVALID, "pb_shell_synth: n_maps must be in [1, 64]");
    if (precision != PB_F32 && precision != PB_F64) return fail(PB_ERR_INVALID, "pb_shell_synth: bad precision");
    SynthParams &p = L->p;
    memset(&p, 0, sizeof(p));
    p.n_maps = n_maps;
    p.n0 = G.n0;
    p.n1 = G.n1;
    p.n2 = G.n2;
    p.nh2 = G.nh2;
    p.m0 = out_n[0];
    p.m1 = out_n[1];
    p.m2 = out_n[2];
    p.kf0 = G.kf0;
    p.kf1 = G.kf1;
    p.kf2 = G.kf2;
    p.los = G.los;
    p.l0 = G.l0;
    p.l1 = G.l1;
    p.l2 = G.l2;
    p.src_stride = src_stride;
    for (int i = 0; i < 3; ++i)
        if (out_n[i] < 2 || (out_n[i] & 1)) return fail(PB_ERR_INVALID, "pb_shell_synth: output dims must be even");
    if (!factor_axis(p.m0, p.ax) || !factor_axis(p.m1, p.ay) || !factor_axis(p.m2, p.az))
        return fail(PB_ERR_UNSUPPORTED, "pb_shell_synth: output dims must be products of 2, 3 and 5");
    const bool f64 = precision == PB_F64;
    const int lx = f64 ? lines_for<double2>(p.m0, 32) : lines_for<float2>(p.m0, 32);
    const int ly = f64 ? lines_for<double2>(p.m1, 32) : lines_for<float2>(p.m1, 32);
    const int lz = f64 ? lines_for<double2>(p.m2, 32) : lines_for<float2>(p.m2, 32);
    auto lg = [](int v) { int k = 0; while ((1 << k) < v) ++k; return k; };
    p.ax.lshift = lg(lx);
    p.ay.lshift = lg(ly);
    p.az.lshift = lg(lz);
    int max_wu = 1;
    for (int m = 0; m < n_maps; ++m) {
        SynthMap &mp = p.maps[m];
        if (!(hi[m] > 0.0) || !std::isfinite(hi[m]))
            return fail(PB_ERR_UNSUPPORTED, "pb_shell_synth: every map needs a finite upper edge");
        if (l1[m] < 0 || l1[m] > 4 || l2[m] < 0 || l2[m] > 4)
            return fail(PB_ERR_INVALID, "pb_shell_synth: Legendre order must be in [0, 4]");
        const int wp = wpow ? wpow[m] : 0;
        if (wp < -1 || wp > 2) return fail(PB_ERR_INVALID, "pb_shell_synth: wpow must be -1, 0, 1 or 2");
        mp.lo = lo[m];
        mp.hi = hi[m];
        mp.scale = scale[m];
        mp.src = src_idx ? src_idx[m] : 0;
        if (mp.src < 0) return fail(PB_ERR_INVALID, "pb_shell_synth: negative source index");
        mp.l1 = l1[m];
        mp.l2 = l2[m];
        mp.wpow = wp;
        // band half-widths with one index of margin (the exact membership test is per mode)
        mp.rx = (int)std::floor(hi[m] / G.kf0) + 1;
        mp.ry = (int)std::floor(hi[m] / G.kf1) + 1;
        mp.kz_max = (int)std::floor(hi[m] / G.kf2) + 1;
        // the band must sit strictly inside the output grid and inside the source grid
        if (2 * mp.rx >= p.m0 || 2 * mp.ry >= p.m1 || 2 * mp.kz_max >= p.m2 || 2 * mp.rx >= G.n0 ||
            2 * mp.ry >= G.n1 || mp.kz_max >= G.nh2 - 1)
            return fail(PB_ERR_UNSUPPORTED, "pb_shell_synth: band limit reaches the Nyquist frequency of a grid");
        mp.wu = 2 * mp.ry + 1;
        max_wu = std::max(max_wu, mp.wu);
    }
    p.c1 = (max_wu + lx - 1) / lx;
    int64_t u = 0, h = 0;
    int b1 = 0, b2 = 0, b3 = 0;
    const int xch = (p.m0 + ly - 1) / ly;
    const int ych = (p.m1 + 2 * lz - 1) / (2 * lz);
    for (int m = 0; m < n_maps; ++m) {
        SynthMap &mp = p.maps[m];
        const int planes = mp.kz_max + 1;
        mp.u_off = u;
        mp.h_off = h;
        u += (int64_t)planes * p.m0 * mp.wu;
        h += (int64_t)planes * p.m0 * p.m1;
        mp.b1 = b1;
        mp.b2 = b2;
        mp.b3 = b3;
        b1 += planes * p.c1;
        b2 += planes * xch;
        b3 += p.m0 * ych;
    }
    L->u_elems = u;
    L->h_elems = h;
    L->nb1 = b1;
    L->nb2 = b2;
    L->nb3 = b3;
    return PB_OK;
}


// dynamic shared memory of a transform kernel
template <typename K>
static cudaError_t set_smem(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Lengths with a compile-time kernel; any other supported length runs the run-time form.
template <typename F>
static void with_length(int n, F &&f) {
    switch (n) {
        case 24: f(std::integral_constant<int, 24>()); break;
        case 32: f(std::integral_constant<int, 32>()); break;
        case 48: f(std::integral_constant<int, 48>()); break;
        case 64: f(std::integral_constant<int, 64>()); break;
        case 96: f(std::integral_constant<int, 96>()); break;
        case 128: f(std::integral_constant<int, 128>()); break;
        case 192: f(std::integral_constant<int, 192>()); break;
        case 256: f(std::integral_constant<int, 256>()); break;
        case 384: f(std::integral_constant<int, 384>()); break;
        case 512: f(std::integral_constant<int, 512>()); break;
        default: f(std::integral_constant<int, 0>()); break;
    }
}

template <typename T, typename S = typename cplx<T>::type>
static int launch_synth(const SynthLayout &L, const S *src, const T *w, typename cplx<T>::type *U,
                        typename cplx<T>::type *H, T *out, cudaStream_t s) {
    const SynthParams &p = L.p;
    const size_t c = sizeof(typename cplx<T>::type);
    auto smem = [&](const FftAxis &a) { return (size_t)(2 * (1 << a.lshift) * (a.n + 1) + a.n) * c; };
    const size_t smem_z = smem(p.az);
    cudaError_t e = cudaSuccess;
    with_length(p.ax.n, [&](auto NC) {
        constexpr int N = decltype(NC)::value;
        if (e == cudaSuccess)
            e = set_smem(synth_x_kernel<T, N, S>, smem(p.ax));
        if (e == cudaSuccess) {
            synth_x_kernel<T, N, S><<<L.nb1, SY_THREADS, smem(p.ax), s>>>(p, src, w, U);
            e = cudaGetLastError();
        }
    });
    if (e != cudaSuccess) return cuda_check(e, "pb_shell_synth (x)");
    with_length(p.ay.n, [&](auto NC) {
        constexpr int N = decltype(NC)::value;
        if (e == cudaSuccess)
            e = set_smem(synth_y_kernel<T, N>, smem(p.ay));
        if (e == cudaSuccess) {
            synth_y_kernel<T, N><<<L.nb2, SY_THREADS, smem(p.ay), s>>>(p, U, H);
            e = cudaGetLastError();
        }
    });
    if (e != cudaSuccess) return cuda_check(e, "pb_shell_synth (y)");
    with_length(p.az.n, [&](auto NC) {
        constexpr int N = decltype(NC)::value;
        if constexpr (std::is_same<T, float>::value && N > 0 && pass_count(N) >= 2) {
            // a tiled set: blocks over groups of maps (rows of neighbouring maps written together)
            const int Lz = 1 << p.az.lshift;
            if (p.tiled && p.m1 % 2 == 0 && Lz >= SY_TMAPS) {
                const int LY = Lz / SY_TMAPS;
                const int64_t nb = (int64_t)p.m0 * ((p.m1 + 2 * LY - 1) / (2 * LY)) *
                                   ((p.n_maps + SY_TMAPS - 1) / SY_TMAPS);
                if (e == cudaSuccess)
                    e = set_smem(synth_z_tiled_kernel<N>, smem_z);
                if (e == cudaSuccess) {
                    synth_z_tiled_kernel<N><<<(unsigned)nb, SY_THREADS_Z, smem_z, s>>>(p, H, reinterpret_cast<char *>(out));
                    e = cudaGetLastError();
                }
                return;
            }
        }
        if (e == cudaSuccess)
            e = set_smem(synth_z_kernel<T, N>, smem_z);
        if (e == cudaSuccess) {
            synth_z_kernel<T, N><<<L.nb3, SY_THREADS_Z, smem_z, s>>>(p, H, out);
            e = cudaGetLastError();
        }
    });
    if (e != cudaSuccess) return cuda_check(e, "pb_shell_synth (z)");
    return PB_OK;
}

}  // namespace pb

using namespace pb;

extern "C" int pb_shell_synth_workspace_size(const pb_grid_t *g, const int32_t *out_n, int precision, int n_maps,
                                             const double *hi, size_t *bytes) {
    if (!bytes || !hi) return fail(PB_ERR_INVALID, "pb_shell_synth_workspace_size: NULL argument");
    if (n_maps < 1 || n_maps > SY_MAX_MAPS)
        return fail(PB_ERR_INVALID, "pb_shell_synth_workspace_size: n_maps must be in [1, 64]");
    if (precision == PB_F32_SRC_F64) precision = PB_F32;  // the workspace holds FP32 transforms
    std::vector<double> lo(n_maps, 0.0), sc(n_maps, 1.0);
    std::vector<int32_t> zero(n_maps, 0);
    SynthLayout L;
    int st = synth_layout(g, out_n, precision, n_maps, lo.data(), hi, nullptr, zero.data(), zero.data(), sc.data(),
                          nullptr, 0, &L);
    if (st) return st;
    const size_t c = precision == PB_F64 ? 16 : 8;
    *bytes = (size_t)(L.u_elems + L.h_elems) * c + 256;
    return PB_OK;
}

static int shell_synth(const pb_grid_t *g, const int32_t *out_n, int precision, const void *src, int64_t src_stride,
                       int n_maps, const int32_t *src_idx, const double *lo, const double *hi, const int32_t *l1,
                       const int32_t *l2, const double *scale, const int32_t *wpow, const void *w, void *out,
                       void *workspace, size_t workspace_bytes, void *stream, bool tiled, int n_factor) {
    if (!out || !lo || !hi || !l1 || !l2 || !scale) return fail(PB_ERR_INVALID, "pb_shell_synth: NULL argument");
    // FP32 maps from a complex FP64 source: only the x pass's reads differ
    const bool src64 = precision == PB_F32_SRC_F64;
    if (src64) precision = PB_F32;
    SynthLayout L;
    int st = synth_layout(g, out_n, precision, n_maps, lo, hi, src_idx, l1, l2, scale, wpow, src_stride, &L);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    if (tiled) {
        if (precision != PB_F32) return fail(PB_ERR_INVALID, "pb_shell_synth_tiled: tiled sets hold f32 maps");
        if ((uintptr_t)out & 15) return fail(PB_ERR_INVALID, "pb_shell_synth_tiled: output not 16-byte aligned");
        if (n_factor < 1 || n_factor > n_maps)
            return fail(PB_ERR_INVALID, "pb_shell_synth_tiled: n_factor must be in [1, n_maps]");
        L.p.tiled = 1;
        L.p.t_maps = n_maps;
        L.p.t_factor = n_factor;
        // the voxels past the grid in the last tile read as zeros (the z pass then writes
        // every voxel of the grid; padding rows are never read)
        const int64_t n_vox = (int64_t)L.p.m0 * L.p.m1 * L.p.m2;
        if (n_vox % TILED_VOX) {
            const int64_t tb = tiled_tile_bytes(n_maps, n_factor);
            PB_CUDA(cudaMemsetAsync((char *)out + (tiled_tiles(n_vox) - 1) * tb, 0, (size_t)tb, s));
        }
    }
    for (int m = 0; m < n_maps; ++m)
        if (L.p.maps[m].wpow != 0 && !w) return fail(PB_ERR_INVALID, "pb_shell_synth: wpow set but weight grid is NULL");
    const size_t c = precision == PB_F64 ? 16 : 8;
    const size_t need = (size_t)(L.u_elems + L.h_elems) * c + 256;
    if (!workspace || workspace_bytes < need) return fail(PB_ERR_INVALID, "pb_shell_synth: workspace too small");
    char *ws = (char *)(((uintptr_t)workspace + 255) & ~(uintptr_t)255);
    if (src64) {
        float2 *U = (float2 *)ws;
        st = launch_synth<float, double2>(L, (const double2 *)src, (const float *)w, U, U + L.u_elems, (float *)out, s);
    } else if (precision == PB_F32) {
        float2 *U = (float2 *)ws;
        st = launch_synth<float>(L, (const float2 *)src, (const float *)w, U, U + L.u_elems, (float *)out, s);
    } else {
        double2 *U = (double2 *)ws;
        st = launch_synth<double>(L, (const double2 *)src, (const double *)w, U, U + L.u_elems, (double *)out, s);
    }
    return st;
}

extern "C" int pb_shell_synth(const pb_grid_t *g, const int32_t *out_n, int precision, const void *src,
                              int64_t src_stride, int n_maps, const int32_t *src_idx, const double *lo,
                              const double *hi, const int32_t *l1, const int32_t *l2, const double *scale,
                              const int32_t *wpow, const void *w, void *out, void *workspace, size_t workspace_bytes,
                              void *stream) {
    return shell_synth(g, out_n, precision, src, src_stride, n_maps, src_idx, lo, hi, l1, l2, scale, wpow, w, out,
                       workspace, workspace_bytes, stream, false, 0);
}

extern "C" int pb_shell_synth_tiled(const pb_grid_t *g, const int32_t *out_n, int precision, const void *src,
                                    int64_t src_stride, int n_maps, int n_factor, const int32_t *src_idx,
                                    const double *lo, const double *hi, const int32_t *l1, const int32_t *l2,
                                    const double *scale, const int32_t *wpow, const void *w, void *out,
                                    void *workspace, size_t workspace_bytes, void *stream) {
    return shell_synth(g, out_n, precision, src, src_stride, n_maps, src_idx, lo, hi, l1, l2, scale, wpow, w, out,
                       workspace, workspace_bytes, stream, true, n_factor);
}
