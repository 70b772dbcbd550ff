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
// n_maps f32 maps of n_vox voxels stored per tile of 128 voxels in the tensor-core
// contraction's staging layout, so that one contiguous copy stages a tile.  The first
// n_factor maps (the pair factors) are kept in FP32; every map is also kept split into bf16
// hi + lo parts, the MMA's operand.  Tile t = [factor slabs][C operand], 512 (F + P) bytes:
//  * factor slabs: 4 slabs of 32 voxels x F rows (F = n_factor rounded up to 8) x 128 bytes,
//    the 16-byte chunk c (voxels 4c..4c+3 of the slab) of row m at chunk position c ^ (m % 8);
//  * C operand: 8 steps of 16 voxels x 2P rows x 32 bytes (P = n_maps rounded up to 16;
//    rows 0..P-1 the hi parts, P..2P-1 the lo parts), the 16-byte half h (voxels 8h..8h+7
//    of the step) of row r at half position h ^ ((r / 4) % 2): the 32-byte-swizzled K-major
//    layout of a tcgen05 operand (8-row atoms of 256 bytes, one MMA K step each), so every
//    MMA reads one contiguous block and 16 voxels of a map are one 32-byte sector.
// Voxels past n_vox hold zeros.
constexpr int TILED_VOX = 128;
__host__ __device__ __forceinline__ int tiled_frows(int n_factor) { return (n_factor + 7) & ~7; }
__host__ __device__ __forceinline__ int tiled_cpad(int n_maps) { return (n_maps + 15) & ~15; }
__host__ __device__ __forceinline__ int64_t tiled_tile_bytes(int n_maps, int n_factor) {
    return 512 * (int64_t)(tiled_frows(n_factor) + tiled_cpad(n_maps));
}
__host__ __device__ __forceinline__ int64_t tiled_tiles(int64_t n_vox) { return (n_vox + TILED_VOX - 1) / TILED_VOX; }
// byte offset of voxel v of factor map m (FP32)
__host__ __device__ __forceinline__ int64_t tiled_factor_byte(int64_t v, int m, int n_maps, int n_factor) {
    const int w = (int)(v & (TILED_VOX - 1));
    return (v >> 7) * tiled_tile_bytes(n_maps, n_factor) + ((w >> 5) * tiled_frows(n_factor) + m) * 128 +
           ((((w & 31) >> 2) ^ (m & 7)) << 4) + (w & 3) * 4;
}
// byte offset of voxel v of C-operand row r (bf16; r < P: hi part of map r, else lo part of map r - P)
__host__ __device__ __forceinline__ int64_t tiled_c_byte(int64_t v, int r, int n_maps, int n_factor) {
    const int w = (int)(v & (TILED_VOX - 1));
    const int P = tiled_cpad(n_maps);
    return (v >> 7) * tiled_tile_bytes(n_maps, n_factor) + 512 * tiled_frows(n_factor) + (w >> 4) * 64 * P +
           (r >> 3) * 256 + (r & 7) * 32 + ((((w & 15) >> 3) ^ ((r >> 2) & 1)) << 4) + (w & 7) * 2;
}

}  // namespace pb
