// Shared device helpers: exact k-grid geometry, Legendre polynomials, error plumbing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include "../../include/polybin3d_b200.h"

namespace pb {

// ---- error plumbing ---------------------------------------------------------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_check(cudaError_t e, const char *where);
#define PB_CUDA(call)                                                   \
    do {                                                                \
        cudaError_t _e = (call);                                        \
        if (_e != cudaSuccess) return ::pb::cuda_check(_e, #call);      \
    } while (0)
#define PB_LAUNCH_CHECK(where)                                          \
    do {                                                                \
        cudaError_t _e = cudaGetLastError();                            \
        if (_e != cudaSuccess) return ::pb::cuda_check(_e, where);      \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

int num_sms();

// launch shapes set through pb_set_tuning (this host thread's settings; zero = default)
const pb_tuning_t &tuning();

// ---- grid geometry ----------------------------------------------------------------
struct Grid {
    int n0, n1, n2, nh2;     // real dims and half-axis length n2/2+1
    double kf0, kf1, kf2;
    int los;                 // 1: mu = (k . (l0, l1, l2)) / |k|, else kz / |k|
    double l0, l1, l2;
    int64_t nhalf;           // n0*n1*nh2
    int64_t nreal;           // n0*n1*n2
};

int make_grid(const pb_grid_t *g, Grid *out);

// frequency index of array position i on an axis of length n (numpy fftshift order)
__device__ __forceinline__ int freq_index(int i, int n) { return i < (n >> 1) ? i : i - n; }

struct Mode {
    double k;    // |k|
    double mu;   // (k . line of sight)/|k| (0 at k=0)
    double deg;  // 1 + (kz > 0)
};

// k . line of sight with the three products summed left to right without FMA, as numpy
// sums them; kz itself for the global (z-axis) line of sight
__device__ __forceinline__ double k_dot_los(int los, double l0, double l1, double l2, double kx, double ky,
                                            double kz) {
    if (!los) return kz;
    return __dadd_rn(__dadd_rn(__dmul_rn(l0, kx), __dmul_rn(l1, ky)), __dmul_rn(l2, kz));
}

// |k| exactly as numpy: k_i = (double)idx*kF_i, sqrt((kx*kx + ky*ky) + kz*kz), no FMA.
__device__ __forceinline__ Mode mode_of(const Grid &g, int64_t idx) {
    int l = (int)(idx % g.nh2);
    int64_t r = idx / g.nh2;
    int j = (int)(r % g.n1);
    int i = (int)(r / g.n1);
    double kx = __dmul_rn((double)freq_index(i, g.n0), g.kf0);
    double ky = __dmul_rn((double)freq_index(j, g.n1), g.kf1);
    double kz = __dmul_rn((double)l, g.kf2);
    double s = __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
    Mode m;
    m.k = __dsqrt_rn(s);
    m.mu = (m.k != 0.0) ? __ddiv_rn(k_dot_los(g.los, g.l0, g.l1, g.l2, kx, ky, kz), m.k) : 0.0;
    m.deg = (l > 0) ? 2.0 : 1.0;
    return m;
}

// Legendre polynomials L_0..L_4 (PolyBin3D/cython/utils.pyx:385-400)
__device__ __forceinline__ double legendre(int l, double mu) {
    double m2 = mu * mu;
    switch (l) {
        case 0: return 1.0;
        case 1: return mu;
        case 2: return 0.5 * (3.0 * m2 - 1.0);
        case 3: return 0.5 * mu * (5.0 * m2 - 3.0);
        default: return (35.0 * m2 * m2 - 30.0 * m2 + 3.0) * 0.125;
    }
}

template <typename T> struct cplx;
template <> struct cplx<float> { using type = float2; };
template <> struct cplx<double> { using type = double2; };

// ---- tiled map sets ---------------------------------------------------------------
// n_maps f32 maps of n_vox voxels as 32-voxel slabs: slab s holds voxels 32 s .. 32 s + 31
// of rows 0 .. R-1 (R = n_maps rounded up to 8), 128 bytes per row, the 16-byte chunk c
// (4 voxels) of row r at chunk position c ^ (r mod 8).  Slabs run to a multiple of 4 (128
// voxels), so any tile of 32, 64 or 128 voxels is one contiguous block laid out as the
// tensor-core contraction stages it in shared memory (the 128-byte swizzle).
constexpr int TILED_SLAB = 32, TILED_ALIGN = 128;
__host__ __device__ __forceinline__ int tiled_rows(int n_maps) { return (n_maps + 7) & ~7; }
__host__ __device__ __forceinline__ int64_t tiled_slabs(int64_t n_vox) {
    return (n_vox + TILED_ALIGN - 1) / TILED_ALIGN * (TILED_ALIGN / TILED_SLAB);
}
// element index of voxel v of map m in a set of `rows` rows
__host__ __device__ __forceinline__ int64_t tiled_index(int64_t v, int m, int rows) {
    const int w = (int)(v & 31);
    return ((v >> 5) * rows + m) * 32 + ((((w >> 2) ^ (m & 7)) << 2) | (w & 3));
}

}  // namespace pb
