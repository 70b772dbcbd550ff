// Tensor-core (tcgen05, sm_100a) triplet contraction
//   out[t] = scale * sum_x A[i1](x) B[i2](x) C[i3](x)
// as the GEMM  D[c_row, pair] = sum_x C_row(x) P_pair(x)  with P_pair = A[i1] * B[i2].
//
// Operands, per tile of TC_KT voxels, in shared memory in the UMMA K-major no-swizzle
// layout (core matrix = 8 rows x 16 B; K chunks LBO apart, padded by 16 B so the producing
// stores are bank-conflict free; 8-row groups 128 B apart):
//   * MMA A = the C maps split into bf16 hi and lo, rows interleaved (row 2j = hi of map j,
//     row 2j + 1 = lo), M = 64 (n_c <= 32) or 128 (n_c <= 64);
//   * MMA B = the pair products split into bf16 hi and lo parts, N <= 256 pairs per tile.
// Per 16-voxel K step and pair tile two MMAs (kind::f16, FP32 accumulate in TMEM),
// C x P_hi and C x P_lo, give all four hi/lo terms; the hi and lo rows of a map sit in
// neighbouring TMEM lanes and are summed with one shuffle when the accumulators are read.
//
// Warp roles (16 warps): producers write the operands from fp32 tiles staged in a ring
// by TMA (cp.async when rows are not 16-byte aligned); one warp stages, one lane issues the
// MMAs; they synchronise through mbarriers only.  Every TC_CHAIN tiles the accumulators are
// folded (tcgen05.ld) into FP64 sums in shared memory, double buffered in TMEM when both
// sets fit.  Every mbarrier wait is bounded; on timeout the CTA records an error in the
// workspace, stops issuing work, drains (bounded) and frees TMEM, and the finalize kernel
// writes NaN outputs.
#include <cuda.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cstring>
#include <string>
#include "pb_triplet.cuh"

namespace pb {

constexpr int TC_KT = 64;                  // voxels per tile (4 MMA K steps of 16)
constexpr int TC_NCHUNK = TC_KT / 8;       // 16-byte K chunks per tile
constexpr int TC_STAGE_LD = TC_KT;         // fp32 staging row stride (elements; TMA box rows are dense)
constexpr int TC_STAGES = 4;               // staging ring depth (tiles in flight per CTA)
#ifndef TC_NBUF
#define TC_NBUF 3
#endif
// operand buffers: producers run TC_NBUF - 1 tiles ahead of the MMAs, which hides the
// commit -> mbarrier -> wake-up round trip of the tensor-core pipe behind operand building
constexpr int TC_OPBUF = TC_NBUF;
constexpr int TC_CHAIN = 16;               // tiles accumulated in TMEM between FP64 folds
constexpr int TC_MAX_NT = 4;               // pair tiles (N <= 256 each)
constexpr int TC_MAX_NC = 64;              // C maps (M = 2 * n_c <= 128)
constexpr long long TC_WAIT_CYCLES = 4000000000LL;  // ~2 s at 2 GHz

struct TcGeom {
    int n_rows;                 // staged map rows
    int off_b, off_c;           // first staged row of the B and C map sets
    int load_b, load_c;         // B / C rows staged from their own pointers (else they lie in A's rows)
    int n_pairs, n_c;
    int M;                      // MMA M: 64 or 128 (C-map rows, hi/lo interleaved)
    int a_lbo, a_bytes;         // C operand: K-chunk stride, bytes per buffer
    int n_nt;                   // pair tiles
    int nt_start[TC_MAX_NT];    // first pair of each tile
    int nt_n[TC_MAX_NT];        // MMA N of each tile (pair count padded)
    int nt_col[TC_MAX_NT];      // TMEM column offset of each tile
    int nt_lbo[TC_MAX_NT];      // K-chunk stride of each tile's operand
    int nt_off[TC_MAX_NT];      // byte offset of each tile's hi part (lo part follows)
    int b_bytes;                // pair operand bytes per buffer
    int ntot;                   // TMEM columns of one accumulator set
    int stage_bytes;
    int tmem_cols, dsets;
    int table_bytes;            // pair table staged in shared memory
    int acc_ld;                 // row stride (doubles) of the FP64 accumulators [n_c][acc_ld], = 2 mod 16
    int acc_bytes;
    int smem_bytes;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    // sm100 shared-memory matrix descriptor: start>>4 [0,14), LBO>>4 [16,30), SBO>>4 [32,46),
    // version 1 [46,48), base offset 0, LBO mode 0, layout SWIZZLE_NONE (0) [61,64)
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int M, int N) {
    // c_format F32 (1) [4,6), a_format BF16 (1) [7,10), b_format BF16 (1) [10,13),
    // K-major A and B, n_dim = N>>3 [17,23), m_dim = M>>4 [24,29)
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

// try_wait with a suspend-time hint: the waiting thread sleeps until the phase completes
// or ~0.1 ms passes, instead of spinning on issue slots the producer warps need
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(100000u)
        : "memory");
    return ok != 0;
}

// bounded wait: false on timeout
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > TC_WAIT_CYCLES) return false;
    }
    return true;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 lanes x 8 columns of 32-bit accumulators; tmem_ld_wait() before the values are used
__device__ __forceinline__ void tmem_ld8_issue(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void cp16(void *smem, const void *gmem, int valid_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem),
                 "r"(valid_bytes));
}
__device__ __forceinline__ void cp4(void *smem, const void *gmem, int valid_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem),
                 "r"(valid_bytes));
}

// split 8 fp32 values into packed bf16 hi and lo parts (hi = rn(x), lo = rn(x - hi))
__device__ __forceinline__ void split8(const float (&x)[8], uint4 &hi, uint4 &lo) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        __nv_bfloat162 hh = __floats2bfloat162_rn(x[2 * i], x[2 * i + 1]);
        float2 hf = __bfloat1622float2(hh);
        __nv_bfloat162 ll = __floats2bfloat162_rn(x[2 * i] - hf.x, x[2 * i + 1] - hf.y);
        h[i] = *reinterpret_cast<uint32_t *>(&hh);
        l[i] = *reinterpret_cast<uint32_t *>(&ll);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

__device__ __forceinline__ void tma_load_2d(void *smem_dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Warp roles: warps 0..TC_PROD-1 produce operands, warp TC_PROD stages tiles (TMA, or
// cp.async), warp TC_PROD+1 issues MMAs, warps TC_FOLD0.. fold the TMEM accumulators of each
// finished chain into the FP64 sums while the producers go on with the next one.
#ifndef TC_NPROD
#define TC_NPROD 14
#endif
#ifndef TC_NUPT
#define TC_NUPT 3
#endif
constexpr int TC_PROD = TC_NPROD;  // producer warps
constexpr int TC_UPT = TC_NUPT;    // units per producer thread handled with hoisted loads
constexpr int TC_FOLDW = 4;        // fold warps, one per TMEM lane quarter
constexpr int TC_THREADS = 32 * (TC_PROD + 2 + TC_FOLDW);
constexpr int TC_LOADW = TC_PROD;  // staging warp
constexpr int TC_MMAW = TC_PROD + 1;
constexpr int TC_FOLD0 = TC_PROD + 2;
static_assert(TC_FOLD0 % 4 == 0, "fold warp w reads TMEM lane quarter w % 4: they must start on a multiple of 4");

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void cp_async_mbar_arrive_noinc(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__global__ void __launch_bounds__(TC_THREADS, 1)
    triplet_tc_kernel(const float *A, int n_a, const float *B, int n_b, const float *C, int n_c, int64_t n_vox,
                      int use_tma, const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                      const __grid_constant__ CUtensorMap map_c, const int32_t *pairs, const __grid_constant__ TcGeom geo,
                      double *partials, int *err) {
    extern __shared__ __align__(128) unsigned char smem[];
    // [FP64 accumulators][stage ring][C operand x2][pair operand x2][pairs]; bases computed
    // arithmetically (runtime-indexed pointer arrays would live in local memory)
    double *const acc = (double *)smem;
    unsigned char *const stage0 = smem + geo.acc_bytes;
    unsigned char *const abuf0 = stage0 + TC_STAGES * geo.stage_bytes;
    unsigned char *const bbuf0 = abuf0 + TC_OPBUF * geo.a_bytes;
    int32_t *const spairs = (int32_t *)(bbuf0 + TC_OPBUF * geo.b_bytes);
    auto stage = [&](int k) { return (float *)(stage0 + k * geo.stage_bytes); };

    __shared__ __align__(8) uint64_t full[TC_STAGES], empty[TC_STAGES];
    __shared__ __align__(8) uint64_t opready[TC_OPBUF], opfree[TC_OPBUF], accready[2], accfree[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t n_tiles = (n_vox + TC_KT - 1) / TC_KT;
    const int64_t my_tiles = n_tiles > blockIdx.x ? (n_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    // operand buffers start at zero: padding rows stay zero for the whole kernel
    for (int i = tid; i < TC_OPBUF * (geo.a_bytes + geo.b_bytes) / 16; i += TC_THREADS)
        reinterpret_cast<uint4 *>(abuf0)[i] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < 2 * geo.n_pairs; i += TC_THREADS) spairs[i] = pairs[i];
    for (int i = tid; i < n_c * geo.acc_ld; i += TC_THREADS) acc[i] = 0.0;
    if (tid == 0) {
        for (int k = 0; k < TC_STAGES; ++k) {
            mbar_init(&full[k], use_tma ? 1 : 32);
            mbar_init(&empty[k], TC_PROD);
        }
        for (int k = 0; k < TC_OPBUF; ++k) {
            mbar_init(&opready[k], TC_PROD);
            mbar_init(&opfree[k], 1);
        }
        for (int k = 0; k < 2; ++k) {
            mbar_init(&accready[k], 1);
            mbar_init(&accfree[k], TC_FOLDW);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                     "r"(geo.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    int last_issued = -1;  // MMA lane: last tile whose MMAs were committed

    if (warp == TC_LOADW) {
        // ---------------- staging warp ----------------
        for (int64_t it = 0; it < my_tiles; ++it) {
            const int slot = (int)(it % TC_STAGES);
            if (it >= TC_STAGES) {
                bool good = true;
                if (lane == 0) good = mbar_wait_bounded(&empty[slot], (uint32_t)(((it - TC_STAGES) / TC_STAGES) & 1));
                good = __shfl_sync(0xffffffffu, good ? 1 : 0, 0) != 0;
                if (!good) { atomicExch(&abort_flag, 1); break; }
            }
            if (*(volatile int *)&abort_flag) break;
            const int64_t v0 = (blockIdx.x + it * (int64_t)gridDim.x) * TC_KT;
            float *dst = stage(slot);
            if (use_tma) {
                if (lane == 0) {
                    mbar_expect_tx(&full[slot], (uint32_t)(geo.n_rows * TC_KT * 4));
                    tma_load_2d(dst, &map_a, (int)v0, 0, &full[slot]);
                    if (geo.load_b) tma_load_2d(dst + geo.off_b * TC_STAGE_LD, &map_b, (int)v0, 0, &full[slot]);
                    if (geo.load_c) tma_load_2d(dst + geo.off_c * TC_STAGE_LD, &map_c, (int)v0, 0, &full[slot]);
                }
            } else {
                for (int e = lane; e < geo.n_rows * TC_KT; e += 32) {
                    int r = e / TC_KT, v = e - r * TC_KT;
                    const float *src;
                    int m;
                    if (r < n_a) { src = A; m = r; }
                    else if (geo.load_b && r < geo.off_b + n_b) { src = B; m = r - geo.off_b; }
                    else { src = C; m = r - geo.off_c; }
                    int64_t x = v0 + v;
                    bool ok = x < n_vox;
                    cp4(dst + r * TC_STAGE_LD + v, src + (int64_t)m * n_vox + (ok ? x : 0), ok ? 4 : 0);
                }
                cp_async_mbar_arrive_noinc(&full[slot]);
            }
        }
    } else if (warp == TC_MMAW) {
        // ---------------- MMA lane ----------------
        if (lane == 0) {
            const uint64_t adesc0 = umma_desc(0, geo.a_lbo, 128);
            int chain = 0, chain_pos = 0;
            for (int64_t it = 0; it < my_tiles; ++it) {
                const int buf = (int)(it % TC_OPBUF);
                if (!mbar_wait_bounded(&opready[buf], (uint32_t)((it / TC_OPBUF) & 1))) {
                    atomicExch(&abort_flag, 1);
                    break;
                }
                if (chain_pos == 0 && chain >= geo.dsets) {
                    const int pc = chain - geo.dsets;
                    if (!mbar_wait_bounded(&accfree[pc % geo.dsets], (uint32_t)((pc / geo.dsets) & 1))) {
                        atomicExch(&abort_flag, 1);
                        break;
                    }
                }
                if (*(volatile int *)&abort_flag) break;
                tc_fence_after();
                const int dset = chain % geo.dsets;
                const uint32_t asm_ = smem_u32(abuf0 + buf * geo.a_bytes);
                const uint32_t bsm = smem_u32(bbuf0 + buf * geo.b_bytes);
                for (int t = 0; t < geo.n_nt; ++t) {
                    const uint32_t d = tmem + (uint32_t)(dset * geo.ntot + geo.nt_col[t]);
                    const uint32_t idesc = umma_idesc_bf16_f32(geo.M, geo.nt_n[t]);
                    const uint64_t bdesc0 = umma_desc(0, geo.nt_lbo[t], 128);
                    const uint32_t bhi = bsm + geo.nt_off[t];
                    const uint32_t part = TC_NCHUNK * geo.nt_lbo[t];
#pragma unroll
                    for (int s2 = 0; s2 < TC_NCHUNK / 2; ++s2) {
                        const uint64_t adesc = adesc0 | (uint64_t)(((asm_ + 2 * s2 * geo.a_lbo) >> 4) & 0x3FFF);
                        const uint32_t bh = bhi + 2 * s2 * geo.nt_lbo[t];
                        const uint64_t dh = bdesc0 | (uint64_t)((bh >> 4) & 0x3FFF);
                        const uint64_t dl = bdesc0 | (uint64_t)(((bh + part) >> 4) & 0x3FFF);
                        umma_bf16(d, adesc, dh, idesc, (chain_pos > 0 || s2 > 0) ? 1u : 0u);
                        umma_bf16(d, adesc, dl, idesc, 1u);
                    }
                }
                umma_commit(&opfree[buf]);
                last_issued = (int)it;
                if (++chain_pos == TC_CHAIN || it + 1 == my_tiles) {
                    umma_commit(&accready[dset]);  // the chain's sums are complete in TMEM
                    chain_pos = 0;
                    ++chain;
                }
            }
        }
    } else if (warp < TC_PROD) {
        // ---------------- producer warps ----------------
        // Units of 8 voxels; K chunk c holds tile voxels {4c..4c+3, 32+4c..32+4c+3} for both
        // operands (the sum over K is order-free), so the 8 lanes of one row read 128
        // contiguous bytes.  Pair units (pair, chunk) first, then C-map units (map, chunk),
        // dealt round-robin; a thread's units are the same every tile, so their offsets
        // are computed once and the TC_UPT units of a tile are loaded before they are
        // converted (the load latencies overlap).
        const int n_unit_p = geo.n_pairs * TC_NCHUNK;
        const int n_unit = n_unit_p + n_c * TC_NCHUNK;
        constexpr int R4 = TC_STAGE_LD / 4;
        constexpr int NPT = 32 * TC_PROD;
        auto unit_info = [&](int u, int &ra, int &rb, int &dst, int &lo, bool &is_pair) {
            const int c = u & (TC_NCHUNK - 1);
            is_pair = u < n_unit_p;
            if (is_pair) {
                const int p = u >> 3;
                ra = spairs[2 * p] * R4 + c;
                rb = (geo.off_b + spairs[2 * p + 1]) * R4 + c;
                int t = 0;
                while (t + 1 < geo.n_nt && p >= geo.nt_start[t + 1]) ++t;
                const int r = p - geo.nt_start[t];
                dst = geo.nt_off[t] + c * geo.nt_lbo[t] + (r >> 3) * 128 + (r & 7) * 16;
                lo = TC_NCHUNK * geo.nt_lbo[t];
            } else {
                const int j = (u - n_unit_p) >> 3;
                ra = (geo.off_c + j) * R4 + c;
                rb = ra;
                const int m = 2 * j;  // hi row; the lo row 2j+1 is the next core-matrix row
                dst = c * geo.a_lbo + (m >> 3) * 128 + (m & 7) * 16;
                lo = 16;
            }
        };
        int u_ra[TC_UPT], u_rb[TC_UPT], u_dst[TC_UPT], u_lo[TC_UPT];
        bool u_ok[TC_UPT], u_pair[TC_UPT];
#pragma unroll
        for (int k = 0; k < TC_UPT; ++k) {
            const int u = tid + k * NPT;
            u_ok[k] = u < n_unit;
            u_ra[k] = u_rb[k] = u_dst[k] = u_lo[k] = 0;
            u_pair[k] = false;
            if (u_ok[k]) unit_info(u, u_ra[k], u_rb[k], u_dst[k], u_lo[k], u_pair[k]);
        }
        for (int64_t it = 0; it < my_tiles; ++it) {
            const int buf = (int)(it % TC_OPBUF);
            const int slot = (int)(it % TC_STAGES);
            bool good = true;
            if (lane == 0) {
                good = mbar_wait_bounded(&full[slot], (uint32_t)((it / TC_STAGES) & 1));
                if (good && it >= TC_OPBUF)
                    good = mbar_wait_bounded(&opfree[buf], (uint32_t)(((it - TC_OPBUF) / TC_OPBUF) & 1));
            }
            good = __shfl_sync(0xffffffffu, good ? 1 : 0, 0) != 0;
            if (!good) { atomicExch(&abort_flag, 1); break; }
            if (*(volatile int *)&abort_flag) break;
            const float4 *st4 = reinterpret_cast<const float4 *>(stage(slot));
            unsigned char *ab = abuf0 + buf * geo.a_bytes;
            unsigned char *bb = bbuf0 + buf * geo.b_bytes;
            float4 va0[TC_UPT], va1[TC_UPT], vb0[TC_UPT], vb1[TC_UPT];
#pragma unroll
            for (int k = 0; k < TC_UPT; ++k) {
                if (u_ok[k]) {
                    va0[k] = st4[u_ra[k]];
                    va1[k] = st4[u_ra[k] + 8];
                    if (u_pair[k]) {
                        vb0[k] = st4[u_rb[k]];
                        vb1[k] = st4[u_rb[k] + 8];
                    } else {
                        vb0[k] = make_float4(1.f, 1.f, 1.f, 1.f);
                        vb1[k] = vb0[k];
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < TC_UPT; ++k) {
                if (!u_ok[k]) continue;
                float x[8] = {va0[k].x * vb0[k].x, va0[k].y * vb0[k].y, va0[k].z * vb0[k].z, va0[k].w * vb0[k].w,
                              va1[k].x * vb1[k].x, va1[k].y * vb1[k].y, va1[k].z * vb1[k].z, va1[k].w * vb1[k].w};
                uint4 hi, lo;
                split8(x, hi, lo);
                unsigned char *dst = (u_pair[k] ? bb : ab) + u_dst[k];
                *reinterpret_cast<uint4 *>(dst) = hi;
                *reinterpret_cast<uint4 *>(dst + u_lo[k]) = lo;
            }
            // units beyond TC_UPT per thread (only for very large pair / map counts)
            for (int u = tid + TC_UPT * NPT; u < n_unit; u += NPT) {
                int ra, rb, dsto, loo;
                bool isp;
                unit_info(u, ra, rb, dsto, loo, isp);
                float4 a0 = st4[ra], a1 = st4[ra + 8];
                float4 b0 = isp ? st4[rb] : make_float4(1.f, 1.f, 1.f, 1.f);
                float4 b1 = isp ? st4[rb + 8] : make_float4(1.f, 1.f, 1.f, 1.f);
                float x[8] = {a0.x * b0.x, a0.y * b0.y, a0.z * b0.z, a0.w * b0.w,
                              a1.x * b1.x, a1.y * b1.y, a1.z * b1.z, a1.w * b1.w};
                uint4 hi, lo;
                split8(x, hi, lo);
                unsigned char *dst = (isp ? bb : ab) + dsto;
                *reinterpret_cast<uint4 *>(dst) = hi;
                *reinterpret_cast<uint4 *>(dst + loo) = lo;
            }
            fence_async_smem();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&empty[slot]);
                mbar_arrive(&opready[buf]);
            }
        }
    }
    if (warp >= TC_FOLD0) {
        // ---------------- fold warps ----------------
        // chain c lives in accumulator set c % dsets; its last MMAs commit accready
        const int q = warp & 3;  // TMEM lane quarter
        // D row held by this lane: M = 64 -> rows 16q..16q+15 in lanes 0..15
        const int m = geo.M == 64 ? (lane < 16 ? 16 * q + lane : -1) : 32 * q + lane;
        const int j = m >= 0 ? (m >> 1) : -1;
        // after the hi + lo shuffle both lanes of a map hold its sums: the hi lane adds the
        // even columns of each group of 8, the lo lane the odd ones; with the accumulator row
        // stride = 2 mod 16 the 16 lanes of one store hit 16 different bank pairs
        const bool writer = m >= 0 && j < n_c;
        const int half = m & 1;
        const int ngrp = geo.ntot / 8;
        const int64_t n_chains = (my_tiles + TC_CHAIN - 1) / TC_CHAIN;
        for (int64_t c = 0; c < n_chains; ++c) {
            const int dset = (int)(c % geo.dsets);
            bool good = true;
            if (lane == 0) good = mbar_wait_bounded(&accready[dset], (uint32_t)((c / geo.dsets) & 1));
            good = __shfl_sync(0xffffffffu, good ? 1 : 0, 0) != 0;
            if (!good) { atomicExch(&abort_flag, 1); break; }
            tc_fence_after();
            const uint32_t tbase = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(dset * geo.ntot);
            for (int cc = 0; cc < ngrp; cc += 2) {
                // two column groups per TMEM wait
                const int cc2 = cc + 1;
                float v[2][8];
                tmem_ld8_issue(tbase + cc * 8, v[0]);
                if (cc2 < ngrp) tmem_ld8_issue(tbase + cc2 * 8, v[1]);
                tmem_ld_wait();
#pragma unroll
                for (int g2 = 0; g2 < 2; ++g2) {
                    const int c8 = cc + g2;
                    if (c8 >= ngrp) break;
#pragma unroll
                    for (int k = 0; k < 8; ++k) v[g2][k] += __shfl_xor_sync(0xffffffffu, v[g2][k], 1);
                    if (writer) {
                        const int col0 = c8 * 8;
                        int t = 0;
                        while (t + 1 < geo.n_nt && col0 >= geo.nt_col[t + 1]) ++t;
                        const int pend = (t + 1 < geo.n_nt) ? geo.nt_start[t + 1] : geo.n_pairs;
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const float val = half ? v[g2][2 * k + 1] : v[g2][2 * k];
                            const int p = geo.nt_start[t] + (col0 + 2 * k + half - geo.nt_col[t]);
                            if (p < pend) acc[j * geo.acc_ld + p] += (double)val;
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&accfree[dset]);
        }
    }
    // ---------------- teardown ----------------
    if (warp == TC_MMAW && lane == 0 && last_issued >= 0) {
        // the MMAs of the last tile must drain before TMEM is freed (bounded)
        mbar_wait_bounded(&opfree[last_issued % TC_OPBUF], (uint32_t)((last_issued / TC_OPBUF) & 1));
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0 && abort_flag) atomicExch(err, PB_ERR_TIMEOUT);
    double *part = partials + (size_t)blockIdx.x * geo.n_pairs * n_c;
    for (int i = tid; i < geo.n_pairs * n_c; i += TC_THREADS) {
        const int p = i / n_c;
        part[i] = acc[(i - p * n_c) * geo.acc_ld + p];
    }
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(geo.tmem_cols));
}

// one warp per triplet: lanes stride over the CTA partials, then a fixed-order warp sum
// (deterministic for a given grid).  Pairs were contracted in chunks of `chunk` pairs: the
// partials of chunk k start at n_cta * k * chunk * n_c, one [pairs of the chunk][n_c] block
// per CTA.
__global__ void triplet_tc_finalize(const double *partials, int n_cta, int n_pairs, int chunk, int n_c,
                                    const int32_t *tmap, int n_trip, double scale, double *out, const int *err) {
    const int t = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= n_trip) return;
    if (*err) {
        if (lane == 0) out[t] = __longlong_as_double(0x7ff8000000000000LL);  // NaN: the contraction timed out
        return;
    }
    const int row = tmap[2 * t], col = tmap[2 * t + 1];
    const int k = row / chunk, p_lo = k * chunk;
    const int pk = min(chunk, n_pairs - p_lo);
    const double *p = partials + (size_t)n_cta * p_lo * n_c + (size_t)(row - p_lo) * n_c + col;
    double s = 0.0;
    for (int c = lane; c < n_cta; c += 32) s += p[(size_t)c * pk * n_c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[t] = s * scale;
}

struct TcRows {
    int n_rows, off_b, off_c, load_b, load_c;
};

static int tc_geometry(const TcRows &rw, int n_pairs, int n_c, TcGeom *g) {
    memset(g, 0, sizeof(*g));
    const int n_rows = rw.n_rows;
    g->n_rows = n_rows;
    g->off_b = rw.off_b;
    g->off_c = rw.off_c;
    g->load_b = rw.load_b;
    g->load_c = rw.load_c;
    g->n_pairs = n_pairs;
    g->n_c = n_c;
    if (n_c > TC_MAX_NC) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: more than 64 C maps");
    g->M = (2 * n_c <= 64) ? 64 : 128;
    g->a_lbo = (g->M / 8) * 128 + 16;
    g->a_bytes = TC_NCHUNK * g->a_lbo;
    const int gran = g->M == 64 ? 8 : 16;  // MMA N granularity
    g->n_nt = (g->n_pairs + 255) / 256;
    if (g->n_nt > TC_MAX_NT) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: more than 1024 pairs");
    int col = 0, off = 0;
    for (int t = 0; t < g->n_nt; ++t) {
        g->nt_start[t] = t * 256;
        int np = std::min(256, g->n_pairs - t * 256);
        g->nt_n[t] = std::max(gran, (np + gran - 1) / gran * gran);
        g->nt_col[t] = col;
        col += g->nt_n[t];
        g->nt_lbo[t] = (g->nt_n[t] / 8) * 128 + 16;
        g->nt_off[t] = off;
        off += 2 * TC_NCHUNK * g->nt_lbo[t];
    }
    g->b_bytes = off;
    g->ntot = col;
    if (g->ntot > 512) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: accumulators exceed TMEM");
    g->dsets = (2 * g->ntot <= 512) ? 2 : 1;
    int cols = 32;
    while (cols < g->dsets * g->ntot) cols *= 2;
    g->tmem_cols = cols;
    g->stage_bytes = n_rows * TC_STAGE_LD * 4;
    g->table_bytes = (int)(2 * g->n_pairs * sizeof(int32_t));
    g->acc_ld = g->n_pairs + (2 - g->n_pairs % 16 + 16) % 16;
    g->acc_bytes = (n_c * g->acc_ld * 8 + 127) / 128 * 128;
    g->smem_bytes = g->acc_bytes + TC_STAGES * g->stage_bytes + TC_OPBUF * (g->a_bytes + g->b_bytes) +
                    (g->table_bytes + 15) / 16 * 16;
    if (g->smem_bytes > 225 * 1024)
        return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: tile too large for shared memory");
    return PB_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point, so the library has no
// link-time dependency on the driver library (it loads on machines without a GPU)
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    static bool looked = false;
    if (!looked) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
        looked = true;
    }
    return fn;
}

static int tc_grid(int64_t n_vox) {
    int64_t n_tiles = (n_vox + TC_KT - 1) / TC_KT;
    return (int)std::max<int64_t>(1, std::min<int64_t>(n_tiles, num_sms()));
}

int triplet_tc_workspace_size(int64_t n_vox, const int32_t *counts, int n_c, size_t *bytes) {
    int gx = tc_grid(n_vox);
    *bytes = 256 + (size_t)gx * counts[1] * n_c * sizeof(double);
    return PB_OK;
}

int launch_triplet_tc(const void *A, int n_a, const void *B, int n_b, const void *C, int n_c, int64_t n_vox,
                      const unsigned char *table, const int32_t *counts, double scale, double *out, void *workspace,
                      size_t workspace_bytes, cudaStream_t s) {
    int dev = 0, major = 0;
    PB_CUDA(cudaGetDevice(&dev));
    PB_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction needs an sm_100 device");
    // staged rows: A's maps, then B's and C's unless they are rows of A already (the same
    // maps, or a contiguous run of them: B = A + k maps) or C is B
    const size_t map_bytes = (size_t)n_vox * 4;
    auto rows_of_a = [&](const void *P, int n_p, int *k) {
        if ((const char *)P < (const char *)A) return false;
        const size_t d = (size_t)((const char *)P - (const char *)A);
        if (d % map_bytes) return false;
        *k = (int)(d / map_bytes);
        return *k + n_p <= n_a && d / map_bytes < (size_t)n_a;
    };
    TcRows rw{n_a, 0, 0, 0, 0};
    if (!rows_of_a(B, n_b, &rw.off_b)) {
        rw.off_b = rw.n_rows;
        rw.load_b = 1;
        rw.n_rows += n_b;
    }
    if (!rows_of_a(C, n_c, &rw.off_c)) {
        if (rw.load_b && C == B && n_c <= n_b) {
            rw.off_c = rw.off_b;
        } else {
            rw.off_c = rw.n_rows;
            rw.load_c = 1;
            rw.n_rows += n_c;
        }
    }
    // pairs go through in chunks small enough for shared memory and TMEM (the FP64
    // accumulators and the pair operands grow with the pair count)
    const int n_pairs = counts[1];
    TcGeom g;
    int chunk = std::min(n_pairs, 512);
    int st = tc_geometry(rw, chunk, n_c, &g);
    while (st == PB_ERR_UNSUPPORTED && chunk > 16 && n_c <= TC_MAX_NC) {
        chunk = (chunk + 1) / 2;
        st = tc_geometry(rw, chunk, n_c, &g);
    }
    if (st) return st;
    int gx = tc_grid(n_vox);
    size_t need = 256 + (size_t)gx * n_pairs * n_c * sizeof(double);
    if (!workspace || workspace_bytes < need)
        return fail(PB_ERR_WORKSPACE, "pb_triplet_contract(tc): workspace too small (need " + std::to_string(need) + ")");
    int *err = (int *)workspace;
    double *partials = (double *)((char *)workspace + 256);
    // TMA staging needs 16-byte aligned rows and at most 256 rows per map set
    int use_tma = ((n_vox % 4) == 0) && (((uintptr_t)A & 15) == 0) && (((uintptr_t)B & 15) == 0) &&
                  (((uintptr_t)C & 15) == 0) && n_a <= 256 && n_b <= 256 && n_c <= 256 && n_vox < (1LL << 31);
    CUtensorMap maps[3];
    memset(maps, 0, sizeof(maps));
    EncodeTiledFn enc = use_tma ? encode_tiled() : nullptr;
    if (!enc) use_tma = 0;
    if (use_tma) {
        const void *bases[3] = {A, B, C};
        const int rows[3] = {n_a, n_b, n_c};
        for (int k = 0; k < 3 && use_tma; ++k) {
            cuuint64_t dims[2] = {(cuuint64_t)n_vox, (cuuint64_t)rows[k]};
            cuuint64_t strides[1] = {(cuuint64_t)n_vox * 4};
            cuuint32_t box[2] = {(cuuint32_t)TC_KT, (cuuint32_t)rows[k]};
            cuuint32_t estr[2] = {1, 1};
            CUresult r = enc(&maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(bases[k]),
                                                dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) use_tma = 0;
        }
    }
    TableLayout L = table_layout(counts);
    PB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    const int32_t *pairs = (const int32_t *)(table + L.off_pairs);
    int smem_max = 0;
    for (int p_lo = 0; p_lo < n_pairs; p_lo += chunk) {
        const int pk = std::min(chunk, n_pairs - p_lo);
        TcGeom gk;
        st = tc_geometry(rw, pk, n_c, &gk);
        if (st) return st;
        if (gk.smem_bytes > smem_max) {
            PB_CUDA(cudaFuncSetAttribute(triplet_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, gk.smem_bytes));
            smem_max = gk.smem_bytes;
        }
        triplet_tc_kernel<<<gx, TC_THREADS, gk.smem_bytes, s>>>(
            (const float *)A, n_a, (const float *)B, n_b, (const float *)C, n_c, n_vox, use_tma, maps[0], maps[1],
            maps[2], pairs + 2 * p_lo, gk, partials + (size_t)gx * p_lo * n_c, err);
        PB_LAUNCH_CHECK("pb_triplet_contract(tc)");
    }
    triplet_tc_finalize<<<(counts[3] + 7) / 8, 256, 0, s>>>(partials, gx, n_pairs, chunk, n_c,
                                                               (const int32_t *)(table + L.off_tmap), counts[3],
                                                               scale, out, err);
    PB_LAUNCH_CHECK("pb_triplet_contract(tc finalize)");
    return PB_OK;
}

}  // namespace pb
