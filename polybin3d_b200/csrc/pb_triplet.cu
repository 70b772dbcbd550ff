// Triplet contraction  out[t] = scale * sum_x A[i1](x) B[i2](x) C[i3](x)  on CUDA cores.
//
// The triplet list is tiled on the host into "items": one A map, up to TB B maps and up
// to TC C maps, so one thread forms TB pair products and TB x TC FMAs per voxel from
// 1 + TB + TC shared-memory loads.  A CTA stages a tile of TV voxels of every map in
// shared memory, P threads share an item (voxels strided by P), per-tile sums are kept in
// the maps' precision and folded into FP64 registers after each tile.  Per-CTA FP64
// partials go to the caller's workspace and a second kernel sums them in a fixed order,
// so results are deterministic.
#include <algorithm>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>
#include <cuda_bf16.h>
#include "pb_common.cuh"
#include "pb_triplet.cuh"

namespace pb {

int triplet_build_items(int n_a, int n_b, int n_c, const int32_t *idx, int n_trip, std::vector<TripletItem> &items) {
    items.clear();
    if (n_trip < 1) return fail(PB_ERR_INVALID, "triplet list is empty");
    if (!idx) return fail(PB_ERR_INVALID, "triplet index array is NULL");
    // a -> list of (b, c, t)
    std::map<int, std::vector<std::array<int, 3>>> by_a;
    std::set<std::array<int, 3>> seen;
    for (int t = 0; t < n_trip; ++t) {
        int a = idx[3 * t], b = idx[3 * t + 1], c = idx[3 * t + 2];
        if (a < 0 || a >= n_a || b < 0 || b >= n_b || c < 0 || c >= n_c)
            return fail(PB_ERR_INVALID, "triplet index out of range at row " + std::to_string(t));
        // each output is written by exactly one work item: a repeated triplet would leave
        // one of its rows unwritten
        if (!seen.insert({a, b, c}).second)
            return fail(PB_ERR_INVALID, "duplicate triplet at row " + std::to_string(t));
        by_a[a].push_back({b, c, t});
    }
    for (auto &kv : by_a) {
        std::vector<int> bs;
        for (auto &e : kv.second) bs.push_back(e[0]);
        std::sort(bs.begin(), bs.end());
        bs.erase(std::unique(bs.begin(), bs.end()), bs.end());
        for (size_t b0 = 0; b0 < bs.size(); b0 += TRIP_TB) {
            size_t nb = std::min<size_t>(TRIP_TB, bs.size() - b0);
            std::vector<int> cs;
            for (auto &e : kv.second)
                for (size_t i = 0; i < nb; ++i)
                    if (e[0] == bs[b0 + i]) cs.push_back(e[1]);
            std::sort(cs.begin(), cs.end());
            cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
            for (size_t c0 = 0; c0 < cs.size(); c0 += TRIP_TC) {
                size_t nc = std::min<size_t>(TRIP_TC, cs.size() - c0);
                TripletItem it;
                it.a = kv.first;
                for (int i = 0; i < TRIP_TB; ++i) it.b[i] = bs[b0 + std::min<size_t>(i, nb - 1)];
                for (int j = 0; j < TRIP_TC; ++j) it.c[j] = cs[c0 + std::min<size_t>(j, nc - 1)];
                for (int i = 0; i < TRIP_TB; ++i)
                    for (int j = 0; j < TRIP_TC; ++j) it.out[i][j] = -1;
                int filled = 0;
                for (auto &e : kv.second) {
                    for (size_t i = 0; i < nb; ++i) {
                        if (e[0] != bs[b0 + i]) continue;
                        for (size_t j = 0; j < nc; ++j)
                            if (e[1] == cs[c0 + j]) {
                                it.out[i][j] = e[2];
                                ++filled;
                            }
                    }
                }
                if (filled) items.push_back(it);
            }
        }
    }
    return PB_OK;
}

// ------------------------------------------------------------------------------------
// SIMT kernel
//
// Tiles of SIMT_TV voxels of every map are staged in shared memory with cp.async, double
// buffered so the next tile's copy overlaps this tile's FMAs.  Per-thread sums stay in
// the maps' precision for SIMT_FLUSH tiles and are then folded into this CTA's FP64
// partial row in global memory (each slot has a single writer, so the order is fixed).
// ------------------------------------------------------------------------------------
constexpr int SIMT_THREADS = 256;
constexpr int SIMT_TV = 128;       // voxels per tile
constexpr int SIMT_PAD = 4;        // row padding (elements) against bank conflicts
constexpr int SIMT_FLUSH = 8;      // tiles between FP64 folds

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int valid_bytes) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

template <typename T>
__device__ __forceinline__ void simt_stage(T *buf, const T *A, int n_a, const T *B, int n_b, int off_b, const T *C,
                                           int off_c, int n_rows, int64_t n_vox, int64_t v0, bool vec) {
    constexpr int LD = SIMT_TV + SIMT_PAD;
    constexpr int EPV = 16 / sizeof(T);  // elements per 16-byte copy
    if (vec) {
        const int per_row = SIMT_TV / EPV;
        for (int e = threadIdx.x; e < n_rows * per_row; e += SIMT_THREADS) {
            int r = e / per_row, c = e - r * per_row;
            const T *src;
            int m;
            if (r < n_a) { src = A; m = r; }
            else if (off_b > 0 && r < off_b + n_b) { src = B; m = r - off_b; }
            else { src = C; m = r - off_c; }
            int64_t x = v0 + (int64_t)c * EPV;
            int64_t left = n_vox - x;
            int bytes = left >= EPV ? 16 : (left > 0 ? (int)left * (int)sizeof(T) : 0);
            const T *g = src + (int64_t)m * n_vox + (bytes > 0 ? x : 0);
            cp_async16(buf + r * LD + c * EPV, g, bytes);
        }
    } else {
        for (int e = threadIdx.x; e < n_rows * SIMT_TV; e += SIMT_THREADS) {
            int r = e / SIMT_TV, v = e - r * SIMT_TV;
            const T *src;
            int m;
            if (r < n_a) { src = A; m = r; }
            else if (off_b > 0 && r < off_b + n_b) { src = B; m = r - off_b; }
            else { src = C; m = r - off_c; }
            int64_t x = v0 + v;
            bool ok = x < n_vox;
            if (sizeof(T) == 4) {
                cp_async4(buf + r * LD + v, src + (int64_t)m * n_vox + (ok ? x : 0), ok);
            } else {
                cp_async4(buf + r * LD + v, src + (int64_t)m * n_vox + (ok ? x : 0), ok);
                cp_async4(reinterpret_cast<char *>(buf + r * LD + v) + 4,
                          reinterpret_cast<const char *>(src + (int64_t)m * n_vox + (ok ? x : 0)) + 4, ok);
            }
        }
    }
    cp_async_commit();
}

template <typename T>
__global__ void __launch_bounds__(SIMT_THREADS, sizeof(T) == 4 ? 3 : 1) triplet_simt_kernel(const T *A, int n_a, const T *B, int n_b,
                                                                      int off_b, const T *C, int n_c, int off_c,
                                                                      int n_rows, int64_t n_vox,
                                                                      const TripletItem *items, int n_items,
                                                                      int group_p, double *partials, int n_trip,
                                                                      int vec) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int LD = SIMT_TV + SIMT_PAD;
    T *buf0 = reinterpret_cast<T *>(smem_raw);
    T *buf1 = buf0 + n_rows * LD;
    const int slots = SIMT_THREADS / group_p;
    const int item_id = blockIdx.y * slots + threadIdx.x / group_p;
    const int p = threadIdx.x % group_p;
    const bool active = item_id < n_items;
    int ra = 0, rb[TRIP_TB], rc[TRIP_TC];
    if (active) {
        // rows clamped into the staged tile: a table built for other map counts cannot
        // index outside shared memory
        const TripletItem &it = items[item_id];
        ra = min(max(it.a, 0), n_rows - 1);
#pragma unroll
        for (int i = 0; i < TRIP_TB; ++i) rb[i] = min(max(off_b + it.b[i], 0), n_rows - 1);
#pragma unroll
        for (int j = 0; j < TRIP_TC; ++j) rc[j] = min(max(off_c + it.c[j], 0), n_rows - 1);
    } else {
#pragma unroll
        for (int i = 0; i < TRIP_TB; ++i) rb[i] = 0;
#pragma unroll
        for (int j = 0; j < TRIP_TC; ++j) rc[j] = 0;
    }
    // output slot of (i, j) in this CTA's partial row, or -1 (read from the table when used)
    const int32_t *outs = active ? &items[item_id].out[0][0] : nullptr;
    double *dst = partials + (int64_t)blockIdx.x * n_trip;
    // this CTA's slots start at zero (single writer per slot: the lane p == 0 of the item)
    if (active && p == 0) {
        for (int q = 0; q < TRIP_TB * TRIP_TC; ++q) {
            int o = outs[q];
            if (o >= 0 && o < n_trip) dst[o] = 0.0;
        }
    }
    T acc[TRIP_TB][TRIP_TC];
#pragma unroll
    for (int i = 0; i < TRIP_TB; ++i)
#pragma unroll
        for (int j = 0; j < TRIP_TC; ++j) acc[i][j] = (T)0;

    const int64_t n_tiles = (n_vox + SIMT_TV - 1) / SIMT_TV;
    int64_t tt = blockIdx.x;
    if (tt < n_tiles) simt_stage<T>(buf0, A, n_a, B, n_b, off_b, C, off_c, n_rows, n_vox, tt * SIMT_TV, vec);
    int cur = 0, since_flush = 0;
    for (; tt < n_tiles; tt += gridDim.x) {
        T *tile = cur ? buf1 : buf0;
        const int64_t nxt = tt + gridDim.x;
        if (nxt < n_tiles) {
            simt_stage<T>(cur ? buf0 : buf1, A, n_a, B, n_b, off_b, C, off_c, n_rows, n_vox, nxt * SIMT_TV, vec);
            cp_async_wait1();
        } else {
            cp_async_wait0();
        }
        __syncthreads();
        if (active) {
            for (int v = p; v < SIMT_TV; v += group_p) {
                T av = tile[ra * LD + v];
                T cv[TRIP_TC];
#pragma unroll
                for (int j = 0; j < TRIP_TC; ++j) cv[j] = tile[rc[j] * LD + v];
#pragma unroll
                for (int i = 0; i < TRIP_TB; ++i) {
                    T pv = av * tile[rb[i] * LD + v];
#pragma unroll
                    for (int j = 0; j < TRIP_TC; ++j) acc[i][j] = fma(pv, cv[j], acc[i][j]);
                }
            }
        }
        __syncthreads();
        cur ^= 1;
        if (++since_flush == SIMT_FLUSH || tt + gridDim.x >= n_tiles) {
            since_flush = 0;
            // reduce over the group_p lanes of an item (consecutive lanes) and fold into FP64
#pragma unroll
            for (int i = 0; i < TRIP_TB; ++i)
#pragma unroll
                for (int j = 0; j < TRIP_TC; ++j) {
                    double s = (double)acc[i][j];
                    for (int o = group_p >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                    if (active && p == 0) {
                        int o = outs[i * TRIP_TC + j];
                        if (o >= 0 && o < n_trip) dst[o] += s;
                    }
                    acc[i][j] = (T)0;
                }
        }
    }
}

__global__ void triplet_finalize(const double *partials, int n_parts, int n_trip, double scale, double *out) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_trip) return;
    double s = 0.0;
    for (int c = 0; c < n_parts; ++c) s += partials[(int64_t)c * n_trip + t];
    out[t] = s * scale;
}

int simt_geometry(int64_t n_vox, int n_items, int *grid_x, int *grid_y, int *group_p) {
    int slots_needed = n_items;
    // threads per item: spread voxels when there are few items
    int p = 1;
    while (p < 32 && (SIMT_THREADS / (p * 2)) >= slots_needed) p *= 2;
    int slots = SIMT_THREADS / p;
    *group_p = p;
    *grid_y = (n_items + slots - 1) / slots;
    int64_t n_tiles = (n_vox + SIMT_TV - 1) / SIMT_TV;
    int64_t gx = std::min<int64_t>(n_tiles, (int64_t)num_sms() * 3);
    *grid_x = (int)std::max<int64_t>(1, gx);
    return PB_OK;
}

int launch_triplet_simt(int precision, const void *A, int n_a, const void *B, int n_b, const void *C, int n_c,
                        int64_t n_vox, const TripletItem *items_dev, int n_items, int n_trip, double scale,
                        double *out, void *workspace, size_t workspace_bytes, cudaStream_t s) {
    int gx, gy, gp;
    simt_geometry(n_vox, n_items, &gx, &gy, &gp);
    size_t need = (size_t)gx * n_trip * sizeof(double);
    if (!workspace || workspace_bytes < need)
        return fail(PB_ERR_WORKSPACE, "pb_triplet_contract: workspace too small (need " + std::to_string(need) + ")");
    int off_b = (B == A && n_b == n_a) ? 0 : n_a;
    int after_b = off_b > 0 ? off_b + n_b : n_a;
    int off_c;
    if (C == A && n_c == n_a) off_c = 0;
    else if (C == B && n_c == n_b) off_c = off_b;
    else off_c = after_b;
    int n_rows = (off_c == after_b) ? after_b + n_c : after_b;
    size_t esz = precision == PB_F64 ? 8 : 4;
    size_t smem = 2 * (size_t)n_rows * (SIMT_TV + SIMT_PAD) * esz;
    if (smem > 227 * 1024) return fail(PB_ERR_UNSUPPORTED, "pb_triplet_contract: too many maps for one tile");
    // 16-byte copies need every map row 16-byte aligned
    size_t align_mask = 15;
    int vec = ((n_vox * (int64_t)esz) % 16 == 0) && (((uintptr_t)A & align_mask) == 0) &&
              (((uintptr_t)B & align_mask) == 0) && (((uintptr_t)C & align_mask) == 0);
    dim3 grid(gx, gy);
    double *partials = (double *)workspace;
    if (precision == PB_F32) {
        PB_CUDA(cudaFuncSetAttribute(triplet_simt_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        triplet_simt_kernel<float><<<grid, SIMT_THREADS, smem, s>>>(
            (const float *)A, n_a, (const float *)B, n_b, off_b, (const float *)C, n_c, off_c, n_rows, n_vox,
            items_dev, n_items, gp, partials, n_trip, vec);
    } else {
        PB_CUDA(cudaFuncSetAttribute(triplet_simt_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        triplet_simt_kernel<double><<<grid, SIMT_THREADS, smem, s>>>(
            (const double *)A, n_a, (const double *)B, n_b, off_b, (const double *)C, n_c, off_c, n_rows, n_vox,
            items_dev, n_items, gp, partials, n_trip, vec);
    }
    PB_LAUNCH_CHECK("pb_triplet_contract(simt)");
    triplet_finalize<<<(n_trip + 255) / 256, 256, 0, s>>>(partials, gx, n_trip, scale, out);
    PB_LAUNCH_CHECK("pb_triplet_contract(finalize)");
    return PB_OK;
}

static size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// plain [n_maps][n_vox] maps -> tiled set (the buffer is zeroed first): one thread per
// (map, voxel), consecutive threads on consecutive voxels of a map (128-byte runs of the
// factor slabs and of the operand rows)
__global__ void tile_maps_kernel(const float *maps, int n_maps, int n_factor, int64_t n_vox, char *out) {
    const int64_t total = (int64_t)n_maps * n_vox;
    const int P = tiled_cpad(n_maps);
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int m = (int)(q / n_vox);
        const int64_t v = q - (int64_t)m * n_vox;
        const float x = maps[q];
        if (m < n_factor) *reinterpret_cast<float *>(out + tiled_factor_byte(v, m, n_maps, n_factor)) = x;
        const __nv_bfloat16 hi = __float2bfloat16_rn(x);
        const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
        *reinterpret_cast<__nv_bfloat16 *>(out + tiled_c_byte(v, m, n_maps, n_factor)) = hi;
        *reinterpret_cast<__nv_bfloat16 *>(out + tiled_c_byte(v, P + m, n_maps, n_factor)) = lo;
    }
}

TableLayout table_layout(const int32_t *counts) {
    TableLayout L;
    L.off_items = 0;
    L.off_pairs = align16(L.off_items + (size_t)counts[0] * sizeof(TripletItem));
    L.off_groups = align16(L.off_pairs + (size_t)counts[1] * 2 * sizeof(int32_t));
    L.off_tmap = align16(L.off_groups + (size_t)counts[2] * sizeof(TcGroup));
    L.bytes = align16(L.off_tmap + (size_t)counts[3] * 2 * sizeof(int32_t));
    return L;
}

}  // namespace pb

using namespace pb;

extern "C" int pb_triplet_plan(int n_a, int n_b, int n_c, const int32_t *idx, int n_trip, void *table,
                               size_t *table_bytes, int32_t *counts) {
    std::vector<TripletItem> items;
    int st = triplet_build_items(n_a, n_b, n_c, idx, n_trip, items);
    if (st) return st;
    // pair rows (i1, i2) in lexicographic order, groups sharing i1, and triplet -> (row, col)
    std::map<std::pair<int, int>, int> pair_row;
    for (int t = 0; t < n_trip; ++t) pair_row[{idx[3 * t], idx[3 * t + 1]}] = 0;
    std::vector<int32_t> pairs;
    int r = 0;
    for (auto &kv : pair_row) {
        kv.second = r++;
        pairs.push_back(kv.first.first);
        pairs.push_back(kv.first.second);
    }
    std::vector<TcGroup> groups;
    for (int row = 0; row < r;) {
        TcGroup g;
        g.a = pairs[2 * row];
        g.row0 = row;
        g.count = 0;
        g.pad = 0;
        while (row < r && g.count < TC_GROUP && pairs[2 * row] == g.a) {
            ++g.count;
            ++row;
        }
        groups.push_back(g);
    }
    std::vector<int32_t> tmap(2 * (size_t)n_trip);
    for (int t = 0; t < n_trip; ++t) {
        tmap[2 * t] = pair_row[{idx[3 * t], idx[3 * t + 1]}];
        tmap[2 * t + 1] = idx[3 * t + 2];
    }
    int32_t c[4] = {(int32_t)items.size(), (int32_t)r, (int32_t)groups.size(), (int32_t)n_trip};
    if (counts) memcpy(counts, c, sizeof(c));
    TableLayout L = table_layout(c);
    if (!table) {
        if (table_bytes) *table_bytes = L.bytes;
        return PB_OK;
    }
    if (!table_bytes || *table_bytes < L.bytes) return fail(PB_ERR_INVALID, "pb_triplet_plan: table buffer too small");
    unsigned char *T = (unsigned char *)table;
    memset(T, 0, L.bytes);
    memcpy(T + L.off_items, items.data(), items.size() * sizeof(TripletItem));
    memcpy(T + L.off_pairs, pairs.data(), pairs.size() * sizeof(int32_t));
    memcpy(T + L.off_groups, groups.data(), groups.size() * sizeof(TcGroup));
    memcpy(T + L.off_tmap, tmap.data(), tmap.size() * sizeof(int32_t));
    *table_bytes = L.bytes;
    return PB_OK;
}

static int check_counts(const int32_t *counts) {
    if (!counts) return fail(PB_ERR_INVALID, "triplet counts are NULL");
    if (counts[0] < 1 || counts[1] < 1 || counts[2] < 1 || counts[3] < 1)
        return fail(PB_ERR_INVALID, "triplet plan is empty");
    return PB_OK;
}

extern "C" int pb_triplet_workspace_size(int precision, int method, int64_t n_vox, const int32_t *counts, int n_c,
                                         size_t *bytes) {
    if (!bytes) return fail(PB_ERR_INVALID, "bytes is NULL");
    int st = check_counts(counts);
    if (st) return st;
    if (n_vox < 1) return fail(PB_ERR_INVALID, "pb_triplet_workspace_size: empty");
    if (precision != PB_F32 && precision != PB_F64) return fail(PB_ERR_INVALID, "bad precision");
    if (method == PB_TRIPLET_TC) return triplet_tc_workspace_size(n_vox, counts, n_c, bytes);
    int gx, gy, gp;
    simt_geometry(n_vox, counts[0], &gx, &gy, &gp);
    *bytes = (size_t)gx * counts[3] * sizeof(double);
    return PB_OK;
}

extern "C" int pb_triplet_contract(int precision, int method, const void *A, int n_a, const void *B, int n_b,
                                   const void *C, int n_c, int64_t n_vox, const void *table, const int32_t *counts,
                                   double scale, double *out, void *workspace, size_t workspace_bytes, void *stream) {
    if (!A || !B || !C || !table || !out) return fail(PB_ERR_INVALID, "pb_triplet_contract: NULL argument");
    int st = check_counts(counts);
    if (st) return st;
    if (n_vox < 1) return fail(PB_ERR_INVALID, "pb_triplet_contract: empty contraction");
    if (n_a < 1 || n_b < 1 || n_c < 1) return fail(PB_ERR_INVALID, "pb_triplet_contract: empty map set");
    if (precision != PB_F32 && precision != PB_F64) return fail(PB_ERR_INVALID, "bad precision");
    const unsigned char *T = (const unsigned char *)table;
    if (method == PB_TRIPLET_TC) {
        if (precision != PB_F32) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction takes f32 maps");
        return launch_triplet_tc(A, n_a, B, n_b, C, n_c, n_vox, T, counts, scale, out, workspace, workspace_bytes,
                                 as_stream(stream));
    }
    if (method != PB_TRIPLET_SIMT) return fail(PB_ERR_INVALID, "bad method");
    TableLayout L = table_layout(counts);
    return launch_triplet_simt(precision, A, n_a, B, n_b, C, n_c, n_vox, (const TripletItem *)(T + L.off_items),
                               counts[0], counts[3], scale, out, workspace, workspace_bytes, as_stream(stream));
}

extern "C" int pb_tiled_maps_bytes(int n_maps, int n_factor, int64_t n_vox, size_t *bytes) {
    if (!bytes) return fail(PB_ERR_INVALID, "pb_tiled_maps_bytes: bytes is NULL");
    if (n_maps < 1 || n_vox < 1) return fail(PB_ERR_INVALID, "pb_tiled_maps_bytes: empty map set");
    if (n_factor < 1 || n_factor > n_maps) return fail(PB_ERR_INVALID, "pb_tiled_maps_bytes: n_factor not in [1, n_maps]");
    *bytes = (size_t)(tiled_tiles(n_vox) * tiled_tile_bytes(n_maps, n_factor));
    return PB_OK;
}

extern "C" int pb_tile_maps(const void *maps, int n_maps, int n_factor, int64_t n_vox, void *tiled, void *stream) {
    if (!maps || !tiled) return fail(PB_ERR_INVALID, "pb_tile_maps: NULL argument");
    if (n_maps < 1 || n_vox < 1) return fail(PB_ERR_INVALID, "pb_tile_maps: empty map set");
    if (n_factor < 1 || n_factor > n_maps) return fail(PB_ERR_INVALID, "pb_tile_maps: n_factor not in [1, n_maps]");
    if ((uintptr_t)tiled & 15) return fail(PB_ERR_INVALID, "pb_tile_maps: output not 16-byte aligned");
    cudaStream_t s = as_stream(stream);
    PB_CUDA(cudaMemsetAsync(tiled, 0, (size_t)(tiled_tiles(n_vox) * tiled_tile_bytes(n_maps, n_factor)), s));
    const int64_t total = (int64_t)n_maps * n_vox;
    const int64_t blocks = std::min<int64_t>((total + 255) / 256, (int64_t)num_sms() * 16);
    tile_maps_kernel<<<(int)blocks, 256, 0, s>>>((const float *)maps, n_maps, n_factor, n_vox, (char *)tiled);
    PB_LAUNCH_CHECK("pb_tile_maps");
    return PB_OK;
}

extern "C" int pb_triplet_contract_tiled(int method, const void *maps, int n_maps, int n_factor, int64_t n_vox,
                                         const void *table, const int32_t *counts, double scale, double *out,
                                         void *workspace, size_t workspace_bytes, void *stream) {
    if (!maps || !table || !out) return fail(PB_ERR_INVALID, "pb_triplet_contract_tiled: NULL argument");
    int st = check_counts(counts);
    if (st) return st;
    if (n_vox < 1 || n_maps < 1) return fail(PB_ERR_INVALID, "pb_triplet_contract_tiled: empty contraction");
    if (n_factor < 1 || n_factor > n_maps)
        return fail(PB_ERR_INVALID, "pb_triplet_contract_tiled: n_factor not in [1, n_maps]");
    if (method != PB_TRIPLET_TC)
        return fail(PB_ERR_UNSUPPORTED, "pb_triplet_contract_tiled: only the tensor-core method reads tiled sets");
    return launch_triplet_tc_tiled((const char *)maps, n_maps, n_factor, n_vox, (const unsigned char *)table, counts,
                                   scale, out, workspace, workspace_bytes, as_stream(stream));
}
