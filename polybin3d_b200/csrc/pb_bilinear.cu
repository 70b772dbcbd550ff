// Bilinear maps: out[o](x) = sum_t [o_t == o] c_t G[i_t](x) G[j_t](x).
//
// The gradient of a weighted sum of triplet sums, sum_t gamma_t sum_x G_a G_b G_c, with
// respect to map G_o is the map sum over the triplets' legs of gamma_t times the product of
// the other two maps; gathering all legs that end on the same output into one real-space
// map leaves one forward transform per output instead of one per (pair of maps).
//
// A block stages a tile of 32 BL_V voxels of every input map in shared memory as
// [map][voxel]; its warps take the outputs round-robin, lane l owning tile voxels l, l+32,
// ..., l+32(BL_V-1) (a warp reads one map at 32 consecutive voxels: one wavefront).  An
// output's terms are sorted by (i, j): per i-group a lane accumulates s = sum_j c G_j, then
// acc += G_i s.  Term records are read by the whole warp at once (a broadcast load) and stay
// in L1 across tiles; four blocks per SM keep enough warps in flight to cover their latency.
#include <algorithm>
#include <tuple>
#include <vector>
#include "pb_common.cuh"

namespace pb {

constexpr int BL_THREADS = 256;
constexpr int BL_MAXG = 128;      // input maps
constexpr int BL_MAXOUT = 4096;   // outputs

// term record: code = j | i << 8 | (first term of an i-group) << 16, the coefficient in
// FP32 and FP64
struct BlTerm {
    uint32_t code;
    float cf;
    double c;
};

template <typename T>
__device__ __forceinline__ T term_coef(const BlTerm &r);
template <>
__device__ __forceinline__ float term_coef<float>(const BlTerm &r) { return r.cf; }
template <>
__device__ __forceinline__ double term_coef<double>(const BlTerm &r) { return r.c; }

// BL_V voxels per lane (8 in FP32, 4 in FP64: the same registers), tile = 32 BL_V voxels
template <typename T, int BL_V>
__global__ void __launch_bounds__(BL_THREADS, 4) bilinear_kernel(const T *G, int n_g, int64_t n_vox,
                                                                 const int32_t *offs, const BlTerm *rec, int n_out,
                                                                 T *out) {
    extern __shared__ __align__(16) unsigned char bl_smem[];
    constexpr int BL_TILE = 32 * BL_V;
    T *sg = reinterpret_cast<T *>(bl_smem);  // [map][BL_TILE]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = BL_THREADS >> 5;
    for (int64_t v0 = (int64_t)blockIdx.x * BL_TILE; v0 < n_vox; v0 += (int64_t)gridDim.x * BL_TILE) {
        __syncthreads();
        for (int e = threadIdx.x; e < n_g * BL_TILE; e += BL_THREADS) {
            const int m = e / BL_TILE, v = e - m * BL_TILE;
            sg[e] = (v0 + v < n_vox) ? G[(int64_t)m * n_vox + v0 + v] : (T)0;
        }
        __syncthreads();
        for (int o = warp; o < n_out; o += nw) {
            T acc[BL_V], s[BL_V], gi[BL_V];
#pragma unroll
            for (int u = 0; u < BL_V; ++u) acc[u] = s[u] = gi[u] = (T)0;
            const int r1 = offs[o + 1];
            for (int r = offs[o]; r < r1; ++r) {
                const BlTerm t = rec[r];
                if (t.code & (1u << 16)) {
#pragma unroll
                    for (int u = 0; u < BL_V; ++u) {
                        acc[u] += gi[u] * s[u];
                        s[u] = (T)0;
                    }
                    const T *gr = sg + ((t.code >> 8) & 0xFF) * BL_TILE + lane;
#pragma unroll
                    for (int u = 0; u < BL_V; ++u) gi[u] = gr[32 * u];
                }
                const T c = term_coef<T>(t);
                const T *gr = sg + (t.code & 0xFF) * BL_TILE + lane;
#pragma unroll
                for (int u = 0; u < BL_V; ++u) s[u] += c * gr[32 * u];
            }
#pragma unroll
            for (int u = 0; u < BL_V; ++u) {
                acc[u] += gi[u] * s[u];
                const int64_t x = v0 + lane + 32 * u;
                if (x < n_vox) out[(int64_t)o * n_vox + x] = acc[u];
            }
        }
    }
}

}  // namespace pb

using namespace pb;

// table: int32 offsets[n_out + 1] (padded to 16 bytes), then the term records of output 0,
// 1, ... each sorted by (i, j) with i <= j and duplicates merged.  An output without terms
// has an empty range and is written as zeros.
extern "C" int pb_bilinear_plan(int n_g, int n_out, const int32_t *o, const int32_t *i, const int32_t *j,
                                const double *c, int n_terms, void *table, size_t *table_bytes, int32_t *n_table) {
    if (!table_bytes || !n_table || (n_terms > 0 && (!o || !i || !j || !c)))
        return fail(PB_ERR_INVALID, "pb_bilinear_plan: NULL argument");
    if (n_g < 1 || n_g > BL_MAXG || n_out < 1 || n_out > BL_MAXOUT)
        return fail(PB_ERR_INVALID, "pb_bilinear_plan: need 1..128 maps and 1..4096 outputs");
    std::vector<std::tuple<int, int, int, double>> t;
    t.reserve(n_terms);
    for (int k = 0; k < n_terms; ++k) {
        if (o[k] < 0 || o[k] >= n_out || i[k] < 0 || i[k] >= n_g || j[k] < 0 || j[k] >= n_g)
            return fail(PB_ERR_INVALID, "pb_bilinear_plan: term index out of range");
        t.emplace_back(o[k], std::min(i[k], j[k]), std::max(i[k], j[k]), c[k]);
    }
    std::sort(t.begin(), t.end(), [](const auto &a, const auto &b) {
        return std::make_tuple(std::get<0>(a), std::get<1>(a), std::get<2>(a)) <
               std::make_tuple(std::get<0>(b), std::get<1>(b), std::get<2>(b));
    });
    std::vector<std::tuple<int, int, int, double>> u;
    for (auto &e : t) {
        if (!u.empty() && std::get<0>(u.back()) == std::get<0>(e) && std::get<1>(u.back()) == std::get<1>(e) &&
            std::get<2>(u.back()) == std::get<2>(e))
            std::get<3>(u.back()) += std::get<3>(e);
        else
            u.push_back(e);
    }
    const int n = (int)u.size();
    const size_t head = ((size_t)(n_out + 1) * 4 + 15) / 16 * 16;
    *table_bytes = head + (size_t)n * sizeof(BlTerm);
    *n_table = n;
    if (!table) return PB_OK;
    int32_t *offs = (int32_t *)table;
    BlTerm *rec = (BlTerm *)((char *)table + head);
    int k = 0;
    for (int q = 0; q < n_out; ++q) {
        offs[q] = k;
        int prev_i = -1;
        while (k < n && std::get<0>(u[k]) == q) {
            const int i_k = std::get<1>(u[k]), j_k = std::get<2>(u[k]);
            rec[k].code = (uint32_t)j_k | ((uint32_t)i_k << 8) | ((uint32_t)(i_k != prev_i) << 16);
            rec[k].cf = (float)std::get<3>(u[k]);
            rec[k].c = std::get<3>(u[k]);
            prev_i = i_k;
            ++k;
        }
    }
    offs[n_out] = k;
    return PB_OK;
}

extern "C" int pb_bilinear_maps(int precision, int64_t n_vox, const void *G, int n_g, const void *table, int n_table,
                                int n_out, void *out, void *stream) {
    if (!G || !table || !out) return fail(PB_ERR_INVALID, "pb_bilinear_maps: NULL argument");
    if (n_vox < 1 || n_g < 1 || n_g > BL_MAXG) return fail(PB_ERR_INVALID, "pb_bilinear_maps: need 1..128 maps");
    if (n_out < 1 || n_out > BL_MAXOUT || n_table < 0)
        return fail(PB_ERR_INVALID, "pb_bilinear_maps: bad output or term count");
    if (((uintptr_t)table & 15) != 0) return fail(PB_ERR_INVALID, "pb_bilinear_maps: table must be 16-byte aligned");
    const bool f64 = precision == PB_F64;
    const int tile = f64 ? 32 * 4 : 32 * 8;
    const size_t smem = (size_t)n_g * tile * (f64 ? 8 : 4);
    const size_t head = ((size_t)(n_out + 1) * 4 + 15) / 16 * 16;
    const int32_t *offs = (const int32_t *)table;
    const BlTerm *rec = (const BlTerm *)((const char *)table + head);
    const int64_t tiles = (n_vox + tile - 1) / tile;
    const int blocks = (int)std::min<int64_t>(tiles, (int64_t)num_sms() * 4 * 8);
    cudaStream_t s = as_stream(stream);
    if (precision == PB_F32) {
        PB_CUDA(cudaFuncSetAttribute(bilinear_kernel<float, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        bilinear_kernel<float, 8><<<blocks, BL_THREADS, smem, s>>>((const float *)G, n_g, n_vox, offs, rec, n_out,
                                                                   (float *)out);
    } else if (precision == PB_F64) {
        PB_CUDA(cudaFuncSetAttribute(bilinear_kernel<double, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        bilinear_kernel<double, 4><<<blocks, BL_THREADS, smem, s>>>((const double *)G, n_g, n_vox, offs, rec, n_out,
                                                                    (double *)out);
    } else {
        return fail(PB_ERR_INVALID, "pb_bilinear_maps: bad precision");
    }
    PB_LAUNCH_CHECK("pb_bilinear_maps");
    return PB_OK;
}
