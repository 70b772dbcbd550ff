// Tensor-core (tcgen05, sm_100a) triplet contraction
//   out[t] = scale * sum_x A[i1](x) B[i2](x) C[i3](x)
// as the GEMM  D[pair, c] = sum_x P_pair(x) C_c(x)  with P_pair = A[i1] * B[i2].
//
// Operands per tile of T voxels (T = 128 by default, 64 or 32 when a shape needs it; K steps of 16):
//   * MMA A = the pair products, in TENSOR MEMORY: one TMEM lane per pair (M = 128 pairs per
//     M-tile, up to TC_MAX_MT M-tiles), split into bf16 hi and lo parts, written by the
//     producer warps with tcgen05.st (two bf16 per 32-bit column, even voxel in the low half);
//   * MMA B = the C maps split into bf16 hi (rows 0..nc_pad-1) and lo (rows nc_pad..), in
//     shared memory in the UMMA K-major no-swizzle layout (core matrix = 8 rows x 16 B, K
//     chunks LBO apart, padded by 16 B so the splitting stores are bank-conflict free).
// Per K step and M-tile two MMAs (kind::f16, FP32 accumulate in TMEM):
//   D[:, 0:2 nc_pad] += P_hi [C_hi; C_lo]^T   and   D[:, 0:nc_pad] += P_lo C_hi^T,
// i.e. the hi*hi, hi*lo and lo*hi terms (lo*lo, ~2^-18 relative, is dropped).  The pair
// products never pass through shared memory: only the staged fp32 map rows (TMA, 128-byte
// swizzle, so that the 32 lanes of a producer warp -- 32 pairs reading up to 8 different
// rows at the same voxels -- hit distinct banks) and the small C operand do.
// Side pairs: when the pair count exceeds a multiple of 128 by at most 16 (the 256^3
// bispectrum's 136 = 128 + 8), the extra pairs do not get a 128-lane M-tile of their own:
// their products go to a small shared-memory operand S (bf16 hi rows, then lo rows) and one
// more MMA per K step, D2[C rows, S rows] += [C_hi; C_lo] S^T (C as the A operand, M = 64 or
// 128), gives all four hi/lo terms.  That keeps the tensor memory for operand buffers and
// the producer work of one lane quarter from doubling.
//
// Staging: from a tiled map set (A = B = C = one set in the slab layout of tiled_index, whose
// tiles are laid out as a stage) each tile is ONE contiguous bulk copy (cp.async.bulk, 16 KB
// for 32 maps at T = 128); from plain [map][voxel] arrays, 32-voxel 2-D TMA boxes of every
// staged row (TMA, or 4-byte cp.async when rows are not 16-byte aligned).  The contiguous copy
// streams at several times the rate of the boxes, whose 128-byte rows are scattered over the
// maps.
// Warp roles (16 warps): 0 stages tiles, 1 issues the MMAs (one lane), 2-3 split the C maps, 4-7 fold accumulators
// (warp w reads TMEM lane quarter w % 4), 8-15 produce pair products (two warps per lane
// quarter, each taking half of a tile's K steps).  They synchronise through mbarriers
// only.  Every `chain` tiles (512 voxels by default) the accumulators are folded
// (tcgen05.ld) into FP64 sums in shared memory, double buffered in TMEM when both sets fit.
// Every mbarrier wait is bounded; on timeout the CTA records an error in the workspace,
// stops issuing work, drains (bounded) and frees TMEM, and the finalize kernel writes NaN
// outputs.
#include <cuda.h>
#include <cuda_bf16.h>
#include <algorithm>
#include <cstring>
#include <string>
#include "pb_triplet.cuh"

namespace pb {

constexpr int TC_MAX_MT = 4;                // pair M-tiles of 128 lanes (<= 512 pairs per launch)
constexpr int TC_MAX_SIDE = 16;             // side pairs (shared-memory operand)
constexpr int TC_MAX_NC = 64;               // C maps per launch
// default voxels accumulated in TMEM between FP64 folds: the tensor core's FP32 accumulation
// loses about half an ulp per K step (measured on positive-mean maps: mean relative error
// -4e-7 after 256 voxels, -9e-7 after 512, -2e-6 after 1024, -5e-6 after 2048)
constexpr int TC_CHAIN_VOX = 512;
constexpr int TC_MAX_STAGES = 6;
constexpr int TC_MAX_NBUF = 4;
constexpr long long TC_WAIT_CYCLES = 4000000000LL;  // ~2 s at 2 GHz

// how a CTA stages its tiles
constexpr int TC_STAGE_CPASYNC = 0, TC_STAGE_TMA = 1, TC_STAGE_TILED = 2;

constexpr int TC_WARPS = 16;
constexpr int TC_THREADS = 32 * TC_WARPS;
constexpr int TC_LOADW = 0, TC_MMAW = 1, TC_CW0 = 2, TC_NCW = 2, TC_FOLD0 = 4, TC_PW0 = 8, TC_PW = 2;
static_assert(TC_FOLD0 % 4 == 0 && TC_PW0 % 4 == 0, "TMEM lane quarter of warp w is w % 4");

struct TcGeom {
    int T;                      // voxels per tile
    int n_rows;                 // staged rows (each loaded set padded to 8 rows)
    int rows_a, rows_b, rows_c; // rows loaded from each set's tensor map (0: the set is rows of another)
    int off_b, off_c;           // first staged row of the B and C maps
    int n_pairs, n_c, nc_pad;   // nc_pad = n_c rounded up to 16 (32 or 64 with side pairs)
    int n_tp;                   // pairs in tensor memory (the first n_tp of the launch)
    int n_mt;                   // pair M-tiles
    int n_side, ns_pad;         // side pairs (after the n_tp) and their operand rows per part (8, 16)
    int side_lbo, side_bytes;   // side operand: K-chunk stride, bytes per buffer
    int d2col0;                 // TMEM column of the side accumulators of set 0 (2 ns_pad per set)
    int acc2_off;               // byte offset of the side FP64 sums [2][n_side][n_c] after acc
    int nstage, nbuf, dsets;
    int pcol0, dcol0, tmem_cols;
    int half_bytes;             // one 32-voxel half of a stage: n_rows x 128 B
    int stage_bytes;
    int cop_lbo, cop_bytes;     // C operand: K-chunk stride, bytes per buffer
    int acc_ld;                 // row stride (doubles) of the FP64 sums [pair][acc_ld], odd
    int acc_bytes;              // rounded to 1024
    int smem_bytes;
    int chain;                  // tiles accumulated in TMEM between FP64 folds
    int poll;                   // 1: the MMA lane and the operand producers poll their barriers
    int n_cons;                 // arrivals per stage / operand buffer: active producer warps + C warps
    int pw_active;              // bit q: pair warps of lane quarter q have pairs
    int split_c;                // 1: the C operand is part of the staged tile (a tiled set), bf16 hi/lo in
                                // the 32-byte-swizzled K-major layout at byte c_off of the stage
    int c_off;
    int pair_lim;               // pair factor rows must lie below this
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

// descriptor of a 32-byte-swizzled K-major operand (8-row atoms of 256 bytes, 256-aligned,
// one atom column = one K step of 16 bf16): LBO unused (1), SBO 256 bytes between 8-row
// atoms, version 1, layout type SWIZZLE_32B (6) [61,64)
__device__ __forceinline__ uint64_t umma_desc_sw32(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(256 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)6 << 61);
}

__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int M, int N) {
    // c_format F32 (1) [4,6), a_format BF16 (1) [7,10), b_format BF16 (1) [10,13),
    // K-major A and B, n_dim = N>>3 [17,23), m_dim = M>>4 [24,29)
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

// try_wait with a suspend-time hint (the thread may sleep until the phase completes)
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}

// non-blocking probe of a phase
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait: false on timeout.  poll != 0: spin on test_wait (the waiter reacts at once;
// used on the operand / MMA path), else a suspending try_wait
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int poll = 0) {
    long long t0 = clock64();
    if (poll) {
        while (!mbar_test_wait(bar, parity)) {
            if (clock64() - t0 > TC_WAIT_CYCLES) return false;
        }
        return true;
    }
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > TC_WAIT_CYCLES) return false;
    }
    return true;
}

// slot of a ring of n buffers and the parity of its current use (no division per tile)
struct Ring {
    int idx = 0, phase = 0;
    __device__ __forceinline__ void next(int n) {
        if (++idx == n) {
            idx = 0;
            phase ^= 1;
        }
    }
};

// lane 0 waits (bounded), the warp learns the outcome
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, int lane, int poll = 0) {
    bool good = true;
    if (lane == 0) good = mbar_wait_bounded(bar, parity, poll);
    return __shfl_sync(0xffffffffu, good ? 1 : 0, 0) != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_mbar_arrive_noinc(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// D (TMEM) (+)= A (TMEM, M = 128 lanes x 16 bf16) x B (shared memory descriptor)^T
__device__ __forceinline__ void umma_ts_bf16(uint32_t d_tmem, uint32_t a_tmem, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 lanes x 8 columns of 32-bit values from registers into TMEM (lane quarter of the warp)
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t (&r)[8]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"r"(taddr),
                 "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// 32 lanes x 16 columns of 32-bit accumulators; tmem_ld_wait() before the values are used
__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ void cp4(uint32_t smem, const void *gmem, int valid_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem), "l"(gmem), "r"(valid_bytes));
}

// contiguous global -> shared copy completing on an mbarrier (both addresses 16-byte
// aligned, size a multiple of 16); no multicast
__device__ __forceinline__ void bulk_load(uint32_t smem_dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_dst),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t smem_dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            smem_dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// bf16 hi = rn(x), lo = rn(x - hi) of two fp32 values, packed (first value in the low half)
__device__ __forceinline__ void split2(float x0, float x1, uint32_t &hi, uint32_t &lo) {
    __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    float2 hf = __bfloat1622float2(h);
    __nv_bfloat162 l = __floats2bfloat162_rn(x0 - hf.x, x1 - hf.y);
    hi = *reinterpret_cast<uint32_t *>(&h);
    lo = *reinterpret_cast<uint32_t *>(&l);
}

// packed fp32x2 arithmetic (one instruction for two lanes' worth of values)
__device__ __forceinline__ unsigned long long f2pack(float a, float b) {
    return ((unsigned long long)__float_as_uint(b) << 32) | __float_as_uint(a);
}
__device__ __forceinline__ unsigned long long fmul2(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long fsub2(unsigned long long a, unsigned long long b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
// bf16 hi = rn(x), lo = rn(x - hi) of a packed pair (first value in the low half)
__device__ __forceinline__ void split2p(unsigned long long x, uint32_t &hi, uint32_t &lo) {
    const float x0 = __uint_as_float((uint32_t)x), x1 = __uint_as_float((uint32_t)(x >> 32));
    __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    hi = *reinterpret_cast<uint32_t *>(&h);
    // the bf16 pair back to fp32: low half << 16, high half masked
    const unsigned long long hf = ((unsigned long long)(hi & 0xFFFF0000u) << 32) | (uint32_t)(hi << 16);
    const unsigned long long r = fsub2(x, hf);
    __nv_bfloat162 l = __floats2bfloat162_rn(__uint_as_float((uint32_t)r), __uint_as_float((uint32_t)(r >> 32)));
    lo = *reinterpret_cast<uint32_t *>(&l);
}
// the products of 4 + 4 voxels of two staged rows, split: hi[0..1], lo[0..1] per float4 pair
__device__ __forceinline__ void prod_split4(const float4 &a, const float4 &b, uint32_t *hi, uint32_t *lo) {
    split2p(fmul2(f2pack(a.x, a.y), f2pack(b.x, b.y)), hi[0], lo[0]);
    split2p(fmul2(f2pack(a.z, a.w), f2pack(b.z, b.w)), hi[1], lo[1]);
}
// 8 staged voxels (two float4) split: hi[0..3], lo[0..3]
__device__ __forceinline__ void split4(const float4 &x0, const float4 &x1, uint32_t *hi, uint32_t *lo) {
    split2p(f2pack(x0.x, x0.y), hi[0], lo[0]);
    split2p(f2pack(x0.z, x0.w), hi[1], lo[1]);
    split2p(f2pack(x1.x, x1.y), hi[2], lo[2]);
    split2p(f2pack(x1.z, x1.w), hi[3], lo[3]);
}

// D (TMEM) (+)= A (shared memory descriptor) x B (shared memory descriptor)^T
__device__ __forceinline__ void umma_ss_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// byte offset of the 16-byte chunk `ch` (4 voxels) of staged row r within a 32-voxel half
// (TMA 128-byte swizzle: chunk index XOR row mod 8)
__device__ __forceinline__ uint32_t stage_off(int r, int ch) { return (uint32_t)r * 128u + (uint32_t)((ch ^ (r & 7)) << 4); }

template <int T>
__global__ void __launch_bounds__(TC_THREADS, 1)
    triplet_tc_kernel(const float *A, int n_a, const float *B, int n_b, const float *C, int n_c, int64_t n_vox,
                      int stage_mode, const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                      const __grid_constant__ CUtensorMap map_c, const int32_t *pairs, const __grid_constant__ TcGeom geo,
                      double *partials, int *err) {
    constexpr int KS = T / 16;       // MMA K steps per tile
    constexpr int HALVES = T / 32;   // 32-voxel swizzled halves per stage
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // [FP64 sums][stage ring][C operand buffers][pair rows], from a 1024-byte boundary of the
    // shared window (the 128-byte swizzle atom of the staged rows)
    unsigned char *const smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    double *const acc = (double *)smem;
    unsigned char *const stage0 = smem + geo.acc_bytes;
    unsigned char *const cop0 = stage0 + geo.nstage * geo.stage_bytes;
    unsigned char *const sop0 = cop0 + geo.nbuf * geo.cop_bytes;
    int32_t *const spairs = (int32_t *)(sop0 + geo.nbuf * geo.side_bytes);
    double *const acc2 = (double *)(smem + geo.acc2_off);  // [2 (C hi / lo rows)][n_side][n_c]

    __shared__ __align__(8) uint64_t full[TC_MAX_STAGES], empty[TC_MAX_STAGES];
    __shared__ __align__(8) uint64_t opready[TC_MAX_NBUF], opfree[TC_MAX_NBUF], accready[2], accfree[2];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t n_tiles = (n_vox + T - 1) / T;
    const int my_tiles = n_tiles > blockIdx.x ? (int)((n_tiles - blockIdx.x + gridDim.x - 1) / gridDim.x) : 0;

    // C operand buffers start at zero (the padding rows nc_pad > n_c stay zero)
    for (int i = tid; i < geo.nbuf * (geo.cop_bytes + geo.side_bytes) / 16; i += TC_THREADS)
        reinterpret_cast<uint4 *>(cop0)[i] = make_uint4(0, 0, 0, 0);
    for (int i = tid; i < 2 * geo.n_side * n_c; i += TC_THREADS) acc2[i] = 0.0;
    int bad_rows = 0;
    for (int i = tid; i < 2 * geo.n_pairs; i += TC_THREADS) {
        spairs[i] = pairs[i];
        bad_rows |= (pairs[i] < 0 || pairs[i] >= geo.pair_lim);
    }
    for (int i = tid; i < geo.n_tp * geo.acc_ld; i += TC_THREADS) acc[i] = 0.0;
    if (tid == 0) {
        for (int k = 0; k < geo.nstage; ++k) {
            mbar_init(&full[k], stage_mode == TC_STAGE_CPASYNC ? 32 : 1);
            mbar_init(&empty[k], geo.split_c ? 1 : geo.n_cons);
        }
        for (int k = 0; k < geo.nbuf; ++k) {
            mbar_init(&opready[k], geo.n_cons);
            mbar_init(&opfree[k], 1);
        }
        for (int k = 0; k < 2; ++k) {
            mbar_init(&accready[k], 1);
            mbar_init(&accfree[k], 4);
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
    // a pair row outside its map set (a plan made for other sets) stops the CTA before any work
    if (__syncthreads_or(bad_rows) && tid == 0) abort_flag = 1;
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;
    int last_issued = -1;  // MMA lane: last tile whose MMAs were committed, its operand buffer and use parity
    int last_buf = 0, last_phase = 0;
    const bool rejected = abort_flag != 0;  // bad pair rows: no role starts

    if (rejected) {
    } else if (warp == TC_LOADW) {
        // ---------------- staging warp ----------------
        Ring st;
        for (int it = 0; it < my_tiles; ++it, st.next(geo.nstage)) {
            const int slot = st.idx;
            if (it >= geo.nstage && !warp_wait(&empty[slot], (uint32_t)(st.phase ^ 1), lane)) {
                atomicExch(&abort_flag, 1);
                break;
            }
            if (*(volatile int *)&abort_flag) break;
            const int64_t v0 = (blockIdx.x + it * (int64_t)gridDim.x) * T;
            const uint32_t dst = smem_u32(stage0 + slot * geo.stage_bytes);
            if (stage_mode == TC_STAGE_TILED) {
                // tile v0 / T of the tiled set: one contiguous block
                if (lane == 0) {
                    mbar_expect_tx(&full[slot], (uint32_t)geo.stage_bytes);
                    bulk_load(dst, reinterpret_cast<const char *>(A) + (v0 / T) * (int64_t)geo.stage_bytes,
                              (uint32_t)geo.stage_bytes, &full[slot]);
                }
            } else if (stage_mode == TC_STAGE_TMA) {
                if (lane == 0) {
                    mbar_expect_tx(&full[slot], (uint32_t)(HALVES * (geo.rows_a + geo.rows_b + geo.rows_c) * 128));
#pragma unroll
                    for (int h = 0; h < HALVES; ++h) {
                        const uint32_t d = dst + h * geo.half_bytes;
                        tma_load_2d(d, &map_a, (int)(v0 + 32 * h), 0, &full[slot]);
                        if (geo.rows_b) tma_load_2d(d + geo.off_b * 128, &map_b, (int)(v0 + 32 * h), 0, &full[slot]);
                        if (geo.rows_c) tma_load_2d(d + geo.off_c * 128, &map_c, (int)(v0 + 32 * h), 0, &full[slot]);
                    }
                }
            } else {
                const int nload = geo.rows_a + geo.rows_b + geo.rows_c;
                for (int e = lane; e < nload * T; e += 32) {
                    const int q = e / T, v = e - q * T;
                    const float *src;
                    int m, r;
                    if (q < geo.rows_a) { src = A; m = q; r = q; }
                    else if (q < geo.rows_a + geo.rows_b) { src = B; m = q - geo.rows_a; r = geo.off_b + m; }
                    else { src = C; m = q - geo.rows_a - geo.rows_b; r = geo.off_c + m; }
                    const int64_t x = v0 + v;
                    const bool ok = x < n_vox;
                    const uint32_t d = dst + (v >> 5) * geo.half_bytes + stage_off(r, (v & 31) >> 2) + (v & 3) * 4;
                    cp4(d, src + (int64_t)m * n_vox + (ok ? x : 0), ok ? 4 : 0);
                }
                cp_async_mbar_arrive_noinc(&full[slot]);
            }
        }
    } else if (warp == TC_MMAW) {
        // ---------------- MMA lane ----------------
        if (lane == 0) {
            const uint32_t idesc_hi = umma_idesc_bf16_f32(128, 2 * geo.nc_pad);
            const uint32_t idesc_lo = umma_idesc_bf16_f32(128, geo.nc_pad);
            int chain = 0, chain_pos = 0;
            Ring bf, st, ds;
            for (int it = 0; it < my_tiles; ++it, bf.next(geo.nbuf), st.next(geo.nstage)) {
                const int buf = bf.idx;
                if (!mbar_wait_bounded(&opready[buf], (uint32_t)bf.phase, geo.poll)) {
                    atomicExch(&abort_flag, 1);
                    break;
                }
                if (chain_pos == 0 && chain >= geo.dsets) {
                    // the fold of the chain that used this accumulator set before
                    if (!mbar_wait_bounded(&accfree[ds.idx], (uint32_t)(ds.phase ^ 1), geo.poll)) {
                        atomicExch(&abort_flag, 1);
                        break;
                    }
                }
                const int slot = st.idx;
                // the C operand of a tiled set is read from the stage itself
                if (geo.split_c && !mbar_wait_bounded(&full[slot], (uint32_t)st.phase, geo.poll)) {
                    atomicExch(&abort_flag, 1);
                    break;
                }
                if (*(volatile int *)&abort_flag) break;
                tc_fence_after();
                const int dset = ds.idx;
                const uint32_t csm = geo.split_c ? smem_u32(stage0 + slot * geo.stage_bytes + geo.c_off)
                                                 : smem_u32(cop0 + buf * geo.cop_bytes);
                // K step ks of the C operand: 16 voxels of every row
                auto cdesc = [&](int ks) -> uint64_t {
                    if (geo.split_c) return umma_desc_sw32(csm + ks * 64 * geo.nc_pad);
                    return umma_desc(csm + 2 * ks * geo.cop_lbo, geo.cop_lbo, 128);
                };
                if (geo.n_side) {
                    const uint32_t d2 = tmem + (uint32_t)(geo.d2col0 + dset * 2 * geo.ns_pad);
                    const uint32_t ssm = smem_u32(sop0 + buf * geo.side_bytes);
                    const uint32_t idesc_s = umma_idesc_bf16_f32(2 * geo.nc_pad, 2 * geo.ns_pad);
#pragma unroll
                    for (int ks = 0; ks < KS; ++ks)
                        umma_ss_bf16(d2, cdesc(ks), umma_desc(ssm + 2 * ks * geo.side_lbo, geo.side_lbo, 128), idesc_s,
                                     (chain_pos > 0 || ks > 0) ? 1u : 0u);
                }
                for (int mt = 0; mt < geo.n_mt; ++mt) {
                    const uint32_t d = tmem + (uint32_t)(geo.dcol0 + (dset * geo.n_mt + mt) * 2 * geo.nc_pad);
                    const uint32_t a = tmem + (uint32_t)(geo.pcol0 + (buf * geo.n_mt + mt) * T);
#pragma unroll
                    for (int ks = 0; ks < KS; ++ks) {
                        const uint64_t bdesc = cdesc(ks);
                        umma_ts_bf16(d, a + 16 * ks, bdesc, idesc_hi, (chain_pos > 0 || ks > 0) ? 1u : 0u);
                        umma_ts_bf16(d, a + 16 * ks + 8, bdesc, idesc_lo, 1u);
                    }
                }
                umma_commit(&opfree[buf]);
                if (geo.split_c) umma_commit(&empty[slot]);  // the stage is free once its MMAs are done
                last_issued = it;
                last_buf = buf;
                last_phase = bf.phase;
                if (++chain_pos == geo.chain || it + 1 == my_tiles) {
                    umma_commit(&accready[dset]);  // the chain's sums are complete in TMEM
                    chain_pos = 0;
                    ++chain;
                    ds.next(geo.dsets);
                }
            }
        }
    } else if (warp >= TC_CW0 && warp < TC_CW0 + TC_NCW) {
        // ---------------- C-map splitting warps ----------------
        // unit (map j, 8-voxel chunk c8): two 16-byte reads of the staged row, bf16 hi to
        // row j and lo to row nc_pad + j of the B operand (K chunk c8)
        const int ct = tid - 32 * TC_CW0;
        const int n_unit = geo.split_c ? 0 : n_c * (T / 8);  // a tiled set carries the split C maps
        const int n_sunit = geo.n_side * (T / 8);
        Ring bf, st;
        for (int it = 0; it < my_tiles; ++it, bf.next(geo.nbuf), st.next(geo.nstage)) {
            const int buf = bf.idx, slot = st.idx;
            if (!warp_wait(&full[slot], (uint32_t)st.phase, lane, geo.poll) ||
                (it >= geo.nbuf && !warp_wait(&opfree[buf], (uint32_t)(bf.phase ^ 1), lane, geo.poll))) {
                atomicExch(&abort_flag, 1);
                break;
            }
            if (*(volatile int *)&abort_flag) break;
            const unsigned char *st = stage0 + slot * geo.stage_bytes;
            unsigned char *cb = cop0 + buf * geo.cop_bytes;
            unsigned char *sb = sop0 + buf * geo.side_bytes;
            // two units per step with both units' shared-memory reads ahead of both units' stores:
            // the stores could alias the next reads as far as the compiler can tell, which would
            // serialise the steps on the read latency; a second unit past the end re-reads the
            // first and is not stored
            constexpr int CS = 32 * TC_NCW;
            for (int u = ct; u < n_unit; u += 2 * CS) {
                // C map j, 8 voxels: bf16 hi to row j, lo to row nc_pad + j of the B operand (K chunk c8)
                const bool two = u + CS < n_unit;
                const int u1 = two ? u + CS : u;
                const int j0 = u / (T / 8), c0 = u - j0 * (T / 8);
                const int j1 = u1 / (T / 8), c1 = u1 - j1 * (T / 8);
                const unsigned char *b0 = st + (c0 >> 2) * geo.half_bytes, *b1 = st + (c1 >> 2) * geo.half_bytes;
                const int r0 = geo.off_c + j0, r1 = geo.off_c + j1;
                const float4 x0 = *reinterpret_cast<const float4 *>(b0 + stage_off(r0, 2 * (c0 & 3)));
                const float4 x1 = *reinterpret_cast<const float4 *>(b0 + stage_off(r0, 2 * (c0 & 3) + 1));
                const float4 y0 = *reinterpret_cast<const float4 *>(b1 + stage_off(r1, 2 * (c1 & 3)));
                const float4 y1 = *reinterpret_cast<const float4 *>(b1 + stage_off(r1, 2 * (c1 & 3) + 1));
                uint32_t h[8], l[8];
                split4(x0, x1, h, l);
                split4(y0, y1, h + 4, l + 4);
                unsigned char *e0 = cb + c0 * geo.cop_lbo + (j0 & 7) * 16;
                *reinterpret_cast<uint4 *>(e0 + (j0 >> 3) * 128) = make_uint4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<uint4 *>(e0 + ((geo.nc_pad + j0) >> 3) * 128) = make_uint4(l[0], l[1], l[2], l[3]);
                if (two) {
                    unsigned char *e1 = cb + c1 * geo.cop_lbo + (j1 & 7) * 16;
                    *reinterpret_cast<uint4 *>(e1 + (j1 >> 3) * 128) = make_uint4(h[4], h[5], h[6], h[7]);
                    *reinterpret_cast<uint4 *>(e1 + ((geo.nc_pad + j1) >> 3) * 128) = make_uint4(l[4], l[5], l[6], l[7]);
                }
            }
            for (int v = ct; v < n_sunit; v += 2 * CS) {
                // side pair sp, 8 voxels: products split, hi to row sp, lo to row ns_pad + sp
                const bool two = v + CS < n_sunit;
                const int v1 = two ? v + CS : v;
                const int s0 = v / (T / 8), c0 = v - s0 * (T / 8);
                const int s1 = v1 / (T / 8), c1 = v1 - s1 * (T / 8);
                const int ra0 = spairs[2 * (geo.n_tp + s0)], rb0 = geo.off_b + spairs[2 * (geo.n_tp + s0) + 1];
                const int ra1 = spairs[2 * (geo.n_tp + s1)], rb1 = geo.off_b + spairs[2 * (geo.n_tp + s1) + 1];
                const unsigned char *b0 = st + (c0 >> 2) * geo.half_bytes, *b1 = st + (c1 >> 2) * geo.half_bytes;
                const int ch0 = 2 * (c0 & 3), ch1 = 2 * (c1 & 3);
                const float4 a00 = *reinterpret_cast<const float4 *>(b0 + stage_off(ra0, ch0));
                const float4 b00 = *reinterpret_cast<const float4 *>(b0 + stage_off(rb0, ch0));
                const float4 a01 = *reinterpret_cast<const float4 *>(b0 + stage_off(ra0, ch0 + 1));
                const float4 b01 = *reinterpret_cast<const float4 *>(b0 + stage_off(rb0, ch0 + 1));
                const float4 a10 = *reinterpret_cast<const float4 *>(b1 + stage_off(ra1, ch1));
                const float4 b10 = *reinterpret_cast<const float4 *>(b1 + stage_off(rb1, ch1));
                const float4 a11 = *reinterpret_cast<const float4 *>(b1 + stage_off(ra1, ch1 + 1));
                const float4 b11 = *reinterpret_cast<const float4 *>(b1 + stage_off(rb1, ch1 + 1));
                uint32_t h[8], l[8];
                prod_split4(a00, b00, h, l);
                prod_split4(a01, b01, h + 2, l + 2);
                prod_split4(a10, b10, h + 4, l + 4);
                prod_split4(a11, b11, h + 6, l + 6);
                unsigned char *e0 = sb + c0 * geo.side_lbo + (s0 & 7) * 16;
                *reinterpret_cast<uint4 *>(e0 + (s0 >> 3) * 128) = make_uint4(h[0], h[1], h[2], h[3]);
                *reinterpret_cast<uint4 *>(e0 + ((geo.ns_pad + s0) >> 3) * 128) = make_uint4(l[0], l[1], l[2], l[3]);
                if (two) {
                    unsigned char *e1 = sb + c1 * geo.side_lbo + (s1 & 7) * 16;
                    *reinterpret_cast<uint4 *>(e1 + (s1 >> 3) * 128) = make_uint4(h[4], h[5], h[6], h[7]);
                    *reinterpret_cast<uint4 *>(e1 + ((geo.ns_pad + s1) >> 3) * 128) = make_uint4(l[4], l[5], l[6], l[7]);
                }
            }
            fence_async_smem();
            __syncwarp();
            if (lane == 0) {
                if (!geo.split_c) mbar_arrive(&empty[slot]);
                mbar_arrive(&opready[buf]);
            }
        }
    } else if (warp >= TC_PW0) {
        // ---------------- pair-product warps ----------------
        // lane quarter q = warp % 4, half g of each tile's K steps; TMEM lane 32 q + lane of
        // M-tile mt holds pair 128 mt + 32 q + lane
        const int q = warp & 3, g = (warp - TC_PW0) >> 2;
        if ((geo.pw_active >> q) & 1) {
            // one copy of the K-step body (the M-tile loop is not unrolled: the role's code stays
            // small next to the other roles'); a lane past the pair count reads row 0 and its
            // TMEM lane is never read out
            const uint32_t tq = tmem + ((uint32_t)(32 * q) << 16);
            const uint32_t half = (uint32_t)geo.half_bytes;
            Ring bf, st;
            for (int it = 0; it < my_tiles; ++it, bf.next(geo.nbuf), st.next(geo.nstage)) {
                const int buf = bf.idx, slot = st.idx;
                if (!warp_wait(&full[slot], (uint32_t)st.phase, lane, geo.poll) ||
                    (it >= geo.nbuf && !warp_wait(&opfree[buf], (uint32_t)(bf.phase ^ 1), lane, geo.poll))) {
                    atomicExch(&abort_flag, 1);
                    break;
                }
                if (*(volatile int *)&abort_flag) break;
                tc_fence_after();
                // this warp's K steps start in slab (g * KS / TC_PW) / 2 of the stage
                const unsigned char *sg = stage0 + slot * geo.stage_bytes + (g * (KS / TC_PW) >> 1) * half;
#pragma unroll 1
                for (int mt = 0; mt < geo.n_mt; ++mt) {
                    const int p0 = 128 * mt + 32 * q;
                    if (p0 >= geo.n_tp) break;
                    const int p = min(p0 + lane, geo.n_tp - 1);
                    const uint32_t ra = (uint32_t)spairs[2 * p], rb = (uint32_t)(geo.off_b + spairs[2 * p + 1]);
                    const uint32_t tcol = tq + (uint32_t)(geo.pcol0 + (buf * geo.n_mt + mt) * T);
#pragma unroll
                    for (int kk = 0; kk < KS / TC_PW; ++kk) {
                        const int ks = g * (KS / TC_PW) + kk;
                        // KS / TC_PW is even (T >= 64) or 1: (ks & 1) and the slab step are compile-time
                        const unsigned char *hb = sg + ((KS / TC_PW) >= 2 ? (kk >> 1) * half : 0u);
                        const int odd = (KS / TC_PW) >= 2 ? (kk & 1) : (ks & 1);
                        uint32_t hi[8], lo[8];
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            const int ch = 4 * odd + c;
                            const float4 a = *reinterpret_cast<const float4 *>(hb + stage_off(ra, ch));
                            const float4 b = *reinterpret_cast<const float4 *>(hb + stage_off(rb, ch));
                            prod_split4(a, b, hi + 2 * c, lo + 2 * c);
                        }
                        tmem_st8(tcol + 16 * ks, hi);
                        tmem_st8(tcol + 16 * ks + 8, lo);
                    }
                }
                tmem_st_wait();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) {
                    if (!geo.split_c) mbar_arrive(&empty[slot]);
                    mbar_arrive(&opready[buf]);
                }
            }
        }
    } else if (warp >= TC_FOLD0 && warp < TC_FOLD0 + 4) {
        // ---------------- fold warps ----------------
        // chain c lives in accumulator set c % dsets; lane quarter q holds pairs 128 mt + 32 q + lane
        const int q = warp & 3;
        const int n_chains = (my_tiles + geo.chain - 1) / geo.chain;
        Ring ds;
        for (int c = 0; c < n_chains; ++c, ds.next(geo.dsets)) {
            const int dset = ds.idx;
            if (!warp_wait(&accready[dset], (uint32_t)ds.phase, lane)) {
                atomicExch(&abort_flag, 1);
                break;
            }
            tc_fence_after();
            if (geo.n_side) {
                // D2 row m (C hi rows m < nc_pad, lo rows after): M = 64 keeps rows 16 q .. 16 q + 15
                // in lanes 0..15 of lane quarter q, M = 128 row 32 q + lane
                const int m = (2 * geo.nc_pad == 64) ? (lane < 16 ? 16 * q + lane : -1) : 32 * q + lane;
                const int h2 = m >= 0 ? m / geo.nc_pad : 0, j = m >= 0 ? m - h2 * geo.nc_pad : 0;
                const uint32_t tb = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(geo.d2col0 + dset * 2 * geo.ns_pad);
                uint32_t v0[16], v1[16];
                tmem_ld16_issue(tb, v0);
                if (geo.ns_pad == 16) tmem_ld16_issue(tb + 16, v1);
                tmem_ld_wait();
                if (m >= 0 && j < n_c) {
                    double *a2 = acc2 + (size_t)h2 * geo.n_side * n_c + j;
#pragma unroll
                    for (int sp = 0; sp < TC_MAX_SIDE; ++sp) {
                        if (sp >= geo.n_side) break;
                        // column sp holds the S_hi products, column ns_pad + sp the S_lo ones
                        const float x_hi = __uint_as_float(v0[sp]);
                        const float x_lo = __uint_as_float(geo.ns_pad == 8 ? v0[(8 + sp) & 15] : v1[sp]);
                        a2[(size_t)sp * n_c] += (double)x_hi + (double)x_lo;
                    }
                }
            }
            for (int mt = 0; mt < geo.n_mt; ++mt) {
                const int p0 = 128 * mt + 32 * q;
                if (p0 >= geo.n_tp) break;
                const int p = p0 + lane;
                double *arow = acc + (size_t)min(p, geo.n_tp - 1) * geo.acc_ld;
                const uint32_t tb = tmem + ((uint32_t)(32 * q) << 16) +
                                    (uint32_t)(geo.dcol0 + (dset * geo.n_mt + mt) * 2 * geo.nc_pad);
                for (int j0 = 0; j0 < geo.nc_pad; j0 += 16) {
                    uint32_t h[16], l[16];
                    tmem_ld16_issue(tb + j0, h);
                    tmem_ld16_issue(tb + geo.nc_pad + j0, l);
                    tmem_ld_wait();
                    if (p < geo.n_tp) {
#pragma unroll
                        for (int k = 0; k < 16; ++k)
                            if (j0 + k < n_c)
                                arow[j0 + k] += (double)__uint_as_float(h[k]) + (double)__uint_as_float(l[k]);
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
        mbar_wait_bounded(&opfree[last_buf], (uint32_t)last_phase);
    }
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0 && abort_flag) atomicExch(err, PB_ERR_TIMEOUT);
    double *part = partials + (size_t)blockIdx.x * geo.n_pairs * n_c;
    for (int i = tid; i < geo.n_pairs * n_c; i += TC_THREADS) {
        const int p = i / n_c, j = i - p * n_c;
        part[i] = p < geo.n_tp ? acc[(size_t)p * geo.acc_ld + j]
                               : acc2[(size_t)(p - geo.n_tp) * n_c + j] +
                                     acc2[(size_t)(geo.n_side + p - geo.n_tp) * n_c + j];
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
    int n_rows, rows_a, rows_b, rows_c, off_b, off_c;
    int tiled;     // 1: one tiled set; n_rows = its factor rows, the C operand in the tile
    int pair_lim;  // pair factor indices must lie below this
};

static int pad8(int x) { return (x + 7) & ~7; }

static int tc_geometry(const TcRows &rw, int n_pairs, int n_c, int T, TcGeom *g) {
    memset(g, 0, sizeof(*g));
    g->T = T;
    g->n_rows = rw.n_rows;
    g->rows_a = rw.rows_a;
    g->rows_b = rw.rows_b;
    g->rows_c = rw.rows_c;
    g->off_b = rw.off_b;
    g->off_c = rw.off_c;
    g->n_pairs = n_pairs;
    g->n_c = n_c;
    if (n_c > TC_MAX_NC) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: more than 64 C maps");
    g->split_c = rw.tiled;
    g->pair_lim = rw.pair_lim;
    if (rw.tiled && T != TILED_VOX) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: tiled sets take 128-voxel tiles");
    const int rem = n_pairs % 128;
    g->n_side = (n_pairs > 128 && rem > 0 && rem <= TC_MAX_SIDE) ? rem : 0;
    // the side MMA takes the C operand as its A operand: M = 2 nc_pad must be 64 or 128 (a tiled
    // set's operand has its own row padding: without a fitting one the side pairs get an M-tile)
    if (rw.tiled) {
        g->nc_pad = tiled_cpad(n_c);
        if (g->nc_pad != 32 && g->nc_pad != 64) g->n_side = 0;
    } else {
        g->nc_pad = g->n_side ? (n_c <= 32 ? 32 : 64) : (n_c + 15) / 16 * 16;
    }
    g->n_tp = n_pairs - g->n_side;
    g->ns_pad = g->n_side <= 8 ? 8 : 16;
    g->n_mt = (g->n_tp + 127) / 128;
    if (g->n_mt > TC_MAX_MT) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: more than 512 pairs");
    // TMEM: nbuf pair-operand buffers (n_mt x T columns each) + dsets accumulator sets
    // (n_mt x 2 nc_pad columns each, plus 2 ns_pad for the side pairs), 512 columns in all
    const int pcols = g->n_mt * T, dcols = g->n_mt * 2 * g->nc_pad + (g->n_side ? 2 * g->ns_pad : 0);
    g->nbuf = 0;
    for (int ds = tuning().tc_dsets == 1 ? 1 : 2; ds >= 1 && !g->nbuf; --ds)
        for (int nb = TC_MAX_NBUF; nb >= 2; --nb)
            if (nb * pcols + ds * dcols <= 512) {
                g->nbuf = nb;
                g->dsets = ds;
                break;
            }
    if (!g->nbuf) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: operands exceed TMEM");
    g->pcol0 = 0;
    g->dcol0 = g->nbuf * pcols;
    g->d2col0 = g->dcol0 + g->dsets * g->n_mt * 2 * g->nc_pad;
    int cols = 32;
    while (cols < g->dcol0 + g->dsets * dcols) cols *= 2;
    g->tmem_cols = cols;
    g->half_bytes = rw.n_rows * 128;
    g->stage_bytes = (T / 32) * g->half_bytes;
    g->cop_lbo = (2 * g->nc_pad / 8) * 128 + 16;
    g->cop_bytes = ((T / 8) * g->cop_lbo + 127) / 128 * 128;
    if (rw.tiled) {
        // [factor slabs][C operand: 8 K steps x 2 nc_pad rows x 32 B], as tiled_tile_bytes
        g->c_off = g->stage_bytes;
        g->stage_bytes += 2 * 2 * g->nc_pad * 128;
        g->cop_bytes = 0;
    }
    g->side_lbo = g->n_side ? (2 * g->ns_pad / 8) * 128 + 16 : 0;
    g->side_bytes = g->n_side ? ((T / 8) * g->side_lbo + 127) / 128 * 128 : 0;
    g->acc_ld = g->nc_pad + 1;
    g->acc2_off = g->n_tp * g->acc_ld * 8;
    g->acc_bytes = (g->acc2_off + 2 * g->n_side * n_c * 8 + 1023) / 1024 * 1024;
    const int table = (2 * n_pairs * 4 + 15) / 16 * 16;
    const int fixed = 1024 + g->acc_bytes + g->nbuf * (g->cop_bytes + g->side_bytes) + table;
    const int budget = 225 * 1024;
    int ns = std::min(TC_MAX_STAGES, (budget - fixed) / std::max(1, g->stage_bytes));
    // a tiled set's stage stays until its MMAs are done: as many as fit
    const int want = tuning().tc_stages > 0 ? tuning().tc_stages
                     : rw.tiled             ? TC_MAX_STAGES
                                            : std::max(2, (64 * 1024) / std::max(1, g->stage_bytes));  // ~64 KB
    ns = std::min(ns, want);
    if (ns < 2) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: tile too large for shared memory");
    g->nstage = ns;
    g->smem_bytes = 1024 + g->acc_bytes + ns * g->stage_bytes + g->nbuf * (g->cop_bytes + g->side_bytes) + table;
    g->pw_active = 0;
    int pw = 0;
    for (int q = 0; q < 4; ++q) {
        bool any = false;
        for (int mt = 0; mt < g->n_mt; ++mt) any = any || (128 * mt + 32 * q < g->n_tp);
        if (any) {
            g->pw_active |= 1 << q;
            pw += TC_PW;
        }
    }
    g->n_cons = pw + TC_NCW;
    g->chain = std::max(1, (tuning().tc_chain > 0 ? tuning().tc_chain : TC_CHAIN_VOX) / T);
    g->poll = tuning().tc_wait == 2 ? 1 : 0;
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
    int64_t n_tiles = (n_vox + 31) / 32;
    return (int)std::max<int64_t>(1, std::min<int64_t>(n_tiles, num_sms()));
}

int triplet_tc_workspace_size(int64_t n_vox, const int32_t *counts, int n_c, size_t *bytes) {
    int gx = tc_grid(n_vox);
    *bytes = 256 + (size_t)gx * counts[1] * n_c * sizeof(double);
    return PB_OK;
}

// The pair chunks, launches and finalize of one contraction whose staged rows `rw` and
// staging mode are set; T0 is the preferred tile (smaller tiles, then smaller pair chunks,
// when a shape does not fit TMEM or shared memory).
static int run_triplet_tc(const float *A, int n_a, const float *B, int n_b, const float *C, int n_c, int64_t n_vox,
                          const TcRows &rw, int stage_mode, const CUtensorMap *maps, int T0,
                          const unsigned char *table, const int32_t *counts, double scale, double *out,
                          void *workspace, size_t workspace_bytes, cudaStream_t s, const char *who) {
    const int n_pairs = counts[1];
    int T = T0;
    TcGeom g;
    int chunk = std::min(n_pairs, 128 * TC_MAX_MT);
    int st = tc_geometry(rw, chunk, n_c, T, &g);
    while (st == PB_ERR_UNSUPPORTED && ((T > 32 && !rw.tiled) || chunk > 16)) {
        if (T > 32 && !rw.tiled) T /= 2;
        else chunk = (chunk + 1) / 2;
        st = tc_geometry(rw, chunk, n_c, T, &g);
    }
    if (st) return st;
    int gx = tc_grid(n_vox);
    size_t need = 256 + (size_t)gx * n_pairs * n_c * sizeof(double);
    if (!workspace || workspace_bytes < need)
        return fail(PB_ERR_WORKSPACE, std::string(who) + ": workspace too small (need " + std::to_string(need) + ")");
    int *err = (int *)workspace;
    double *partials = (double *)((char *)workspace + 256);
    TableLayout L = table_layout(counts);
    PB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    const int32_t *pairs = (const int32_t *)(table + L.off_pairs);
    auto kernel_of = [](int t) {
        return t == 128 ? triplet_tc_kernel<128> : (t == 64 ? triplet_tc_kernel<64> : triplet_tc_kernel<32>);
    };
    int smem_max = 0;
    for (int p_lo = 0; p_lo < n_pairs; p_lo += chunk) {
        const int pk = std::min(chunk, n_pairs - p_lo);
        TcGeom gk;
        st = tc_geometry(rw, pk, n_c, T, &gk);
        if (st) return st;
        if (gk.smem_bytes > smem_max) {
            PB_CUDA(cudaFuncSetAttribute(kernel_of(T), cudaFuncAttributeMaxDynamicSharedMemorySize, gk.smem_bytes));
            smem_max = gk.smem_bytes;
        }
        kernel_of(T)<<<gx, TC_THREADS, gk.smem_bytes, s>>>(A, n_a, B, n_b, C, n_c, n_vox, stage_mode, maps[0],
                                                           maps[1], maps[2], pairs + 2 * p_lo, gk,
                                                           partials + (size_t)gx * p_lo * n_c, err);
        PB_LAUNCH_CHECK(who);
    }
    triplet_tc_finalize<<<(counts[3] + 7) / 8, 256, 0, s>>>(partials, gx, n_pairs, chunk, n_c,
                                                               (const int32_t *)(table + L.off_tmap), counts[3],
                                                               scale, out, err);
    PB_LAUNCH_CHECK(who);
    return PB_OK;
}

static int check_device() {
    int dev = 0, major = 0;
    PB_CUDA(cudaGetDevice(&dev));
    PB_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
    if (major != 10) return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction needs an sm_100 device");
    return PB_OK;
}

int launch_triplet_tc(const void *A, int n_a, const void *B, int n_b, const void *C, int n_c, int64_t n_vox,
                      const unsigned char *table, const int32_t *counts, double scale, double *out, void *workspace,
                      size_t workspace_bytes, cudaStream_t s) {
    int st = check_device();
    if (st) return st;
    if (n_a > 256 || n_b > 256 || n_c > TC_MAX_NC)
        return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: more than 256 maps in a set");
    // staged rows: A's maps, then B's and C's unless they are rows of A already (the same
    // maps, or a contiguous run of them: B = A + k maps) or C is B; each loaded set starts
    // on a multiple of 8 rows (1024 bytes per 32-voxel half: the swizzle atom)
    const size_t map_bytes = (size_t)n_vox * 4;
    auto rows_of_a = [&](const void *P, int n_p, int *k) {
        if ((const char *)P < (const char *)A) return false;
        const size_t d = (size_t)((const char *)P - (const char *)A);
        if (d % map_bytes) return false;
        *k = (int)(d / map_bytes);
        return *k + n_p <= n_a && d / map_bytes < (size_t)n_a;
    };
    TcRows rw{pad8(n_a), n_a, 0, 0, 0, 0, 0, std::max(n_a, n_b)};
    if (!rows_of_a(B, n_b, &rw.off_b)) {
        rw.off_b = rw.n_rows;
        rw.rows_b = n_b;
        rw.n_rows += pad8(n_b);
    }
    if (!rows_of_a(C, n_c, &rw.off_c)) {
        if (rw.rows_b && C == B && n_c <= n_b) {
            rw.off_c = rw.off_b;
        } else {
            rw.off_c = rw.n_rows;
            rw.rows_c = n_c;
            rw.n_rows += pad8(n_c);
        }
    }
    // TMA staging needs 16-byte aligned rows
    int stage_mode = ((n_vox % 4) == 0) && (((uintptr_t)A & 15) == 0) && (((uintptr_t)B & 15) == 0) &&
                             (((uintptr_t)C & 15) == 0) && n_vox < (1LL << 31)
                         ? TC_STAGE_TMA
                         : TC_STAGE_CPASYNC;
    CUtensorMap maps[3];
    memset(maps, 0, sizeof(maps));
    EncodeTiledFn enc = stage_mode == TC_STAGE_TMA ? encode_tiled() : nullptr;
    if (!enc) stage_mode = TC_STAGE_CPASYNC;
    if (stage_mode == TC_STAGE_TMA) {
        const void *bases[3] = {A, B, C};
        const int rows[3] = {n_a, n_b, n_c};
        for (int k = 0; k < 3 && stage_mode == TC_STAGE_TMA; ++k) {
            cuuint64_t dims[2] = {(cuuint64_t)n_vox, (cuuint64_t)rows[k]};
            cuuint64_t strides[1] = {(cuuint64_t)n_vox * 4};
            cuuint32_t box[2] = {32u, (cuuint32_t)rows[k]};
            cuuint32_t estr[2] = {1, 1};
            CUresult r = enc(&maps[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void *>(bases[k]), dims, strides,
                             box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) stage_mode = TC_STAGE_CPASYNC;
        }
    }
    // 128-voxel tiles halve the per-tile barrier rounds against 64 (0.91 against 1.07 ms at 32 maps
    // on 192^3); the geometry steps down when a shape does not fit TMEM or shared memory
    const int T = tuning().tc_tile ? tuning().tc_tile : 128;
    return run_triplet_tc((const float *)A, n_a, (const float *)B, n_b, (const float *)C, n_c, n_vox, rw, stage_mode,
                          maps, T, table, counts, scale, out, workspace, workspace_bytes, s, "pb_triplet_contract(tc)");
}

int launch_triplet_tc_tiled(const char *maps, int n_maps, int n_factor, int64_t n_vox, const unsigned char *table,
                            const int32_t *counts, double scale, double *out, void *workspace, size_t workspace_bytes,
                            cudaStream_t s) {
    int st = check_device();
    if (st) return st;
    if (n_maps > TC_MAX_NC)
        return fail(PB_ERR_UNSUPPORTED, "tensor-core contraction: more than 64 maps in a tiled set");
    if ((uintptr_t)maps & 15) return fail(PB_ERR_INVALID, "pb_triplet_contract_tiled: maps not 16-byte aligned");
    // A = B = C = the set: the staged factor rows are its first n_factor maps, the C operand
    // (all maps) comes with the tile
    const TcRows rw{tiled_frows(n_factor), n_factor, 0, 0, 0, 0, 1, n_factor};
    CUtensorMap none[3];
    memset(none, 0, sizeof(none));
    const float *f = reinterpret_cast<const float *>(maps);
    return run_triplet_tc(f, n_maps, f, n_maps, f, n_maps, n_vox, rw, TC_STAGE_TILED, none, TILED_VOX, table, counts,
                          scale, out, workspace, workspace_bytes, s, "pb_triplet_contract_tiled");
}

}  // namespace pb
