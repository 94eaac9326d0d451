// M2L per translation class on the 5th-generation tensor cores (tcgen05),
// split-FP32 ("3xTF32") with FP32 accumulation in tensor memory.
//
// Same contract as m2l.cu (one dense operator T_c per class, applied to the
// gathered source multipoles of a tile of target boxes), with each FP64
// operand x split as x ~ hi + lo, hi = tf32(x), lo = tf32(x - hi), and
//     T*M ~ T_hi*M_hi + T_hi*M_lo + T_lo*M_hi
// (the split-precision scheme of Ootomo & Yokota, "Recovering single
// precision accuracy from Tensor Cores while surpassing the FP32
// theoretical peak performance", 2022), accumulated in FP32 over all
// group (one class) of the tile, and summed over the groups in FP64.
// Long FP32 accumulation chains in the tensor cores lose far more than
// round-to-nearest FP32 would (measured: ~1e-5 relative after ~190 groups
// against ~3e-7 when each group is drained to FP64), hence one
// accumulation session per group.
//
// CTA = 384 threads, one work item: a range of class groups of one output
// tile of 128 coefficient rows x 128 target slots (the MMA is M=128, N=128,
// K=8 per instruction). Operand tiles are K-major and swizzled: each row (a
// coefficient row of T_c, or the coefficients of one source multipole)
// holds TC_KC fp32 of K (16 in 64 bytes, or 32 in 128 bytes, with the
// swizzle of that width); 8 rows form a swizzle atom. K is streamed in
// chunks of TC_KC through a ring of shared-memory stages (6 of 32 KB, or 3
// of 64 KB): a TMA tiled load per operator plane and cp.async row copies of
// the gathered source multipoles, all completing on the stage's "full"
// mbarrier (TMA byte count plus one arrival per loader warp, made once the
// warp's cp.async group for the stage has landed). One thread issues the MMAs of a chunk (TC_KC / 8 K-steps x 3
// products) and commits them to the stage's "empty" mbarrier, which the
// loader waits on before refilling the stage. Every load fills this CTA's own shared memory only. All waits are bounded by a clock
// budget; on expiry the kernel records an error in *status, lets work in
// flight finish, frees its tensor memory and returns.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace sumpy {
namespace {

constexpr int TC_TW = 128;      // target slots per tile (MMA N)
constexpr int TC_M = 128;       // coefficient rows per CTA (MMA M)
#ifndef SUMPY_TC_KC
#define SUMPY_TC_KC 32
#endif
// K per stage: 32 fp32 (128-byte operand rows and swizzle, three stages) or
// 16 (64-byte rows and swizzle, six stages in the same shared memory;
// measured 1.5x slower on the 1M-point M2L: twice the per-stage barrier and
// issue overhead for the same bytes)
constexpr int TC_KC = SUMPY_TC_KC;
static_assert(TC_KC == 16 || TC_KC == 32, "K per stage");
constexpr int ROWB = 4 * TC_KC;                // bytes per operand row = swizzle span
constexpr int CPR = ROWB / 16;                 // 16-byte chunks per row
constexpr int TC_STAGES = TC_KC == 32 ? 3 : 6;
#ifndef SUMPY_TC_GATHER
#define SUMPY_TC_GATHER 0
#endif
// the gathered source rows: cp.async 16-byte copies by three loader warps
// (0), or TMA gather4 by one loader warp (1: same results, measured 3x
// slower on the 1M-point M2L -- 64 gather instructions of 512 bytes per
// stage queue on the SM's one TMA unit)
constexpr bool TC_GATHER = SUMPY_TC_GATHER != 0;
constexpr int TC_LOADERS = 96;             // warps 0-2
constexpr int TC_DRAINERS = 256;           // warps 4-11
constexpr int TC_THREADS = 128 + TC_DRAINERS;
constexpr int PLANE = TC_M * ROWB;         // bytes of one 128-row operand tile
constexpr int STAGE = 4 * PLANE;           // A_hi, A_lo, B_hi, B_lo
constexpr int TC_SMEM = TC_STAGES * STAGE + 1024 /* alignment slack */ + 256 /* barriers */;
static_assert(TC_SMEM <= 227 * 1024, "shared memory per CTA");
constexpr uint32_t TMEM_COLS = 256;         // two 128-column accumulators
// (the budget of every wait is wait_cycles_budget(), common.cuh)
// budgets below this poll the barrier without suspending the thread, so that
// a short budget is measured in cycles rather than in hardware suspend windows
constexpr long long SHORT_WAIT = 1000000LL;

enum { ST_TIMEOUT_MMA = 1 };

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// wait until at most N of this thread's committed cp.async groups are pending
template <int N> __device__ __forceinline__ void cp_async_wait_group()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// make this thread's shared-memory writes visible to the tensor cores (async proxy)
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t addr, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(addr), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_test_wait(uint32_t addr, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, ROWB-byte swizzle (layout
// type 2 = 128-byte, 4 = 64-byte), 8-row atoms 8 * ROWB bytes apart (stride
// byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t sw_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3fff);
    d |= (uint64_t)1 << 16;                 // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)((8 * ROWB) >> 4) << 32; // stride byte offset
    d |= (uint64_t)1 << 46;                 // version
    d |= (uint64_t)(ROWB == 128 ? 2 : 4) << 61;
    return d;
}

// Instruction descriptors: D f32, A/B tf32 (format 2) or f16 (format 0),
// both K-major, N = 128, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_TW >> 3) << 17) |
                           ((uint32_t)(TC_M >> 4) << 24);
constexpr uint32_t IDESC_F16 = (1u << 4) | ((uint32_t)(TC_TW >> 3) << 17) |
                               ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t acc)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t acc)
{
    const uint32_t z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(IDESC_F16), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

struct TcArgs {
    int n, k_pad;
    const int32_t *item_tile, *item_g0, *item_g1;
    const int32_t *tile_targets;
    const double *tile_scale;
    const int32_t *group_class, *group_sources;
    const void *src_hi, *src_lo;       // operand planes (fp32 for tf32, f16 for f16)
    const float *src_rinv, *mat_rinv;  // f16 form: 2^-e of each source row / operator row
    int32_t rows_pad;
    int32_t a_rows;             // operator rows per TMA box: n when it fits one block of 128
    int32_t src_row_base, zero_row;
    int32_t tbase;
    double *tgt;
    int32_t *status;
    long long wait_cycles;      // budget of each barrier wait (clock64 cycles)
};

__device__ __forceinline__ void mbar_arrive(uint32_t addr)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(addr) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t addr, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(addr), "r"(bytes)
                 : "memory");
}

// TMA: one 3D tile (TC_KC fp32 of K x 128 rows x 1 class) of a class-operator plane
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, uint32_t mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(mbar)
        : "memory");
}

// TMA gather of four rows (r0..r3, one row high box of TC_KC fp32 at column
// c0) of a 2D plane into four consecutive swizzled smem rows
__device__ __forceinline__ void tma_gather4(uint32_t dst, const CUtensorMap *map, int c0, int r0,
                                            int r1, int r2, int r3, uint32_t mbar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(r0), "r"(r1), "r"(r2), "r"(r3),
        "r"(mbar)
        : "memory");
}

// bounded wait that also gives up when another thread has aborted
__device__ bool mbar_wait_or_abort(uint32_t addr, uint32_t parity, volatile int *abort_flag,
                                   long long limit)
{
    const long long t0 = clock64();
    const bool poll = limit < SHORT_WAIT;
    while (!(poll ? mbar_test_wait(addr, parity) : mbar_try_wait(addr, parity))) {
        if (*abort_flag) return false;
        if (clock64() - t0 > limit) {
            *abort_flag = 1;
            return false;
        }
    }
    return true;
}

// One CTA per work item = a contiguous range of class groups of one tile.
// Warp roles: warps 0-2 load (thread 0 also posts the expected TMA bytes),
// warp 3 lane 0 issues the MMAs, warps 4-11 drain. Each group's product accumulates in one of
// two TMEM accumulators (128 columns each) and is drained into FP64
// registers right after the group, while the next group accumulates in the
// other: no FP32 sum spans more than one group. Draining warp w covers TMEM
// lanes 32*(w%4).. and 64 of the 128 columns. The item's sums are added to
// the local expansions with FP64 atomics (a tile may span several items).
template <bool F16>
__global__ void __launch_bounds__(TC_THREADS, 1)
m2l_tc_kernel(TcArgs a, const __grid_constant__ CUtensorMap map_a_hi,
                  const __grid_constant__ CUtensorMap map_a_lo,
                  const __grid_constant__ CUtensorMap map_b_hi,
                  const __grid_constant__ CUtensorMap map_b_lo)
{
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_addr(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;          // 1024-byte aligned stages
    uint8_t *base_ptr = smem_raw + (base - raw);
    uint64_t *bars = reinterpret_cast<uint64_t *>(base_ptr + TC_STAGES * STAGE);
    // bars: [0,S) stage full, [S,2S) stage empty, 2S..2S+1 accumulator full,
    // 2S+2..2S+3 accumulator empty
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * TC_STAGES + 4);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
    const uint32_t bar0 = smem_addr(bars);
    const uint32_t full_bar = bar0, empty_bar = bar0 + 8 * TC_STAGES;
    const uint32_t accf_bar = bar0 + 16 * TC_STAGES, acce_bar = accf_bar + 16;

    // operand element size and K per stage (one ROWB-byte row of K)
    constexpr int ES = F16 ? 2 : 4;
    constexpr int KC = ROWB / ES;
    constexpr bool GATHER = TC_GATHER && !F16;
    const int item = blockIdx.x;
    const int row0 = blockIdx.y * TC_M;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_addr(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 32) {
        for (int s = 0; s < TC_STAGES; ++s) {
            // TMA expect-tx + one arrival per copying loader warp
            mbar_init(full_bar + 8 * s, GATHER ? 1 : TC_LOADERS / 32 + 1);
            mbar_init(empty_bar + 8 * s, 1);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(accf_bar + 8 * s, 1);
            mbar_init(acce_bar + 8 * s, TC_DRAINERS / 32);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (threadIdx.x == 64) {
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&map_a_hi)) : "memory");
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&map_a_lo)) : "memory");
        if (GATHER) {
            asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&map_b_hi)) : "memory");
            asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&map_b_lo)) : "memory");
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int tile = a.item_tile[item];
    const int g0 = a.item_g0[item], g1 = a.item_g1[item];
    const int ng = g1 - g0;
    // split K: CTA z of gridDim.z takes K chunks [kcb, kcb + nkc) of every
    // group (the host keeps gridDim.z <= the number of chunks)
    const int nkc_all = a.k_pad / KC;
    const int kcb = (int)((int64_t)blockIdx.z * nkc_all / gridDim.z);
    const int nkc = (int)((int64_t)(blockIdx.z + 1) * nkc_all / gridDim.z) - kcb;
    const int total = ng * nkc;

    if (GATHER && warp == 0) {
        // ---------------- loader (one warp, all TMA) ----------------
        // lane 0: the two operator tiles; lane l: gather4 of slots 4l..4l+3
        // of both source planes (empty slots read the zero row); lane 0
        // posts the stage's bytes once. A group's rows and class are read
        // once per group, one group ahead.
        const unsigned FULL = 0xffffffffu;
        int32_t r_cur[4], r_nxt[4];
        auto load_rows = [&](int g, int32_t *dst) {
            const int32_t *gs = a.group_sources + (int64_t)g * TC_TW + 4 * lane;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int32_t sb = gs[i];
                dst[i] = sb >= 0 ? sb - a.src_row_base : a.zero_row;
            }
        };
        int cls_cur = 0, cls_nxt = 0;
        if (ng > 0) {
            load_rows(g0, r_cur);
            if (lane == 0) cls_cur = a.group_class[g0];
        }
        for (int it = 0; it < total; ++it) {
            const int s = it % TC_STAGES, use = it / TC_STAGES;
            const int gi = it / nkc, kc = it % nkc;
            if (kc == 0 && gi + 1 < ng) {
                load_rows(g0 + gi + 1, r_nxt);
                if (lane == 0) cls_nxt = a.group_class[g0 + gi + 1];
            }
            bool ok = true;
            if (use > 0) ok = mbar_wait_or_abort(empty_bar + 8 * s, (use - 1) & 1, abort_flag, a.wait_cycles);
            if (__any_sync(FULL, !ok || *abort_flag)) break;
            const int k0 = (kcb + kc) * KC;
            const uint32_t st = base + s * STAGE;
            if (lane == 0) {
                mbar_expect_tx(full_bar + 8 * s, 2 * a.a_rows * ROWB + 2 * PLANE);
                tma_load_3d(st, &map_a_hi, k0, row0, cls_cur, full_bar + 8 * s);
                tma_load_3d(st + PLANE, &map_a_lo, k0, row0, cls_cur, full_bar + 8 * s);
            }
            __syncwarp();
            const uint32_t rows4 = (uint32_t)lane * 4 * ROWB;
            tma_gather4(st + 2 * PLANE + rows4, &map_b_hi, k0, r_cur[0], r_cur[1], r_cur[2],
                        r_cur[3], full_bar + 8 * s);
            tma_gather4(st + 3 * PLANE + rows4, &map_b_lo, k0, r_cur[0], r_cur[1], r_cur[2],
                        r_cur[3], full_bar + 8 * s);
            if (kc == nkc - 1) {
#pragma unroll
                for (int i = 0; i < 4; ++i) r_cur[i] = r_nxt[i];
                cls_cur = cls_nxt;
            }
        }
    } else if (!GATHER && warp < TC_LOADERS / 32) {
        // ---------------- loaders ----------------
        // thread 0: TMA tiles of the two operator planes; all 96 threads:
        // cp.async row copies of the two source planes (the gathered
        // multipoles), then an asynchronous arrival on the stage barrier.
        // A thread's (slot, 16-byte column) chunks are c = tid + 96 u; the
        // group's source boxes of those slots are loaded once per group, one
        // group ahead (the same rows serve all K chunks of the group).
        constexpr int NU = (TC_TW * CPR + TC_LOADERS - 1) / TC_LOADERS;
        int32_t sb_cur[NU], sb_nxt[NU];
        auto load_rows = [&](int g, int32_t *dst) {
            const int32_t *gs = a.group_sources + (int64_t)g * TC_TW;
#pragma unroll
            for (int u = 0; u < NU; ++u) {
                const int c = threadIdx.x + u * TC_LOADERS;
                dst[u] = c < TC_TW * CPR ? gs[c / CPR] : -1;
            }
        };
        // thread 0 also reads the group's class (the operator for the TMA
        // loads) one group ahead
        int cls_cur = 0, cls_nxt = 0;
        if (ng > 0) {
            load_rows(g0, sb_cur);
            if (threadIdx.x == 0) cls_cur = a.group_class[g0];
        }
        // Each warp commits a stage's copies as one cp.async group and
        // announces the stage one iteration later, once the group has landed
        // (wait_group 1: all but the newest group): one arrival per warp
        // instead of one per thread keeps the barrier's serialised arrivals
        // off the critical path.
        const unsigned FULLMASK = 0xffffffffu;
        int pending = -1;   // stage whose copies this warp issued but has not announced
        for (int it = 0; it < total; ++it) {
            const int s = it % TC_STAGES, use = it / TC_STAGES;
            const int gi = it / nkc, kc = it % nkc;
            if (kc == 0 && gi + 1 < ng) {
                load_rows(g0 + gi + 1, sb_nxt);
                if (threadIdx.x == 0) cls_nxt = a.group_class[g0 + gi + 1];
            }
            bool ok = true;
            if (use > 0) ok = mbar_wait_or_abort(empty_bar + 8 * s, (use - 1) & 1, abort_flag, a.wait_cycles);
            if (__any_sync(FULLMASK, !ok || *abort_flag)) break;
            const int k0 = (kcb + kc) * KC;
            const uint32_t st = base + s * STAGE;
            if (threadIdx.x == 0) {
                mbar_expect_tx(full_bar + 8 * s, 2 * a.a_rows * ROWB);
                tma_load_3d(st, &map_a_hi, k0, row0, cls_cur, full_bar + 8 * s);
                tma_load_3d(st + PLANE, &map_a_lo, k0, row0, cls_cur, full_bar + 8 * s);
            }
#pragma unroll
            for (int u = 0; u < NU; ++u) {
                const int c = threadIdx.x + u * TC_LOADERS;
                // f16 form: an empty slot's rows are not written at all (the
                // drain skips its columns, whose source scale is zero)
                if (c < TC_TW * CPR && (!F16 || sb_cur[u] >= 0)) {
                    const int slot = c / CPR, q = c % CPR;
                    const int32_t sb = sb_cur[u];
                    // the swizzle: 16-byte chunk q of a row XOR address bits 7.. of the row
                    const uint32_t dst =
                        slot * ROWB + ((q ^ (((slot * ROWB) >> 7) & (CPR - 1))) << 4);
                    // empty slots: zero-fill without reading memory (source size 0)
                    const int64_t row = sb >= 0 ? sb - a.src_row_base : a.zero_row;
                    const int64_t off = (row * a.k_pad + k0) * ES + 16 * q;   // bytes
                    const uint32_t bytes = sb >= 0 ? 16u : 0u;
                    cp_async16(st + 2 * PLANE + dst,
                               static_cast<const char *>(a.src_hi) + off, bytes);
                    cp_async16(st + 3 * PLANE + dst,
                               static_cast<const char *>(a.src_lo) + off, bytes);
                }
            }
            cp_async_commit();
            if (pending >= 0) {
                cp_async_wait_group<1>();
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(full_bar + 8 * pending);
            }
            pending = s;
            if (kc == nkc - 1) {
#pragma unroll
                for (int u = 0; u < NU; ++u) sb_cur[u] = sb_nxt[u];
                cls_cur = cls_nxt;
            }
        }
        // the last stage (and, after an abort, every copy still in flight)
        cp_async_wait_group<0>();
        if (pending >= 0) {
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(full_bar + 8 * pending);
        }
    } else if (warp == 3) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            for (int it = 0; it < total; ++it) {
                const int s = it % TC_STAGES, use = it / TC_STAGES;
                if (!mbar_wait_or_abort(full_bar + 8 * s, use & 1, abort_flag, a.wait_cycles)) break;
                const int gi = it / nkc, kc = it % nkc;
                const int acc = gi & 1;
                if (kc == 0 && gi >= 2 &&
                    !mbar_wait_or_abort(acce_bar + 8 * acc, ((gi >> 1) - 1) & 1, abort_flag, a.wait_cycles))
                    break;
                tc_fence_after();
                const uint32_t st = base + s * STAGE;
                const uint64_t ah = sw_desc(st), al = sw_desc(st + PLANE);
                const uint64_t bh = sw_desc(st + 2 * PLANE), bl = sw_desc(st + 3 * PLANE);
                const uint32_t d = tmem + (uint32_t)(acc * TC_TW);
#pragma unroll
                for (int k = 0; k < ROWB / 32; ++k) {
                    // one MMA K-step is 32 bytes along K (8 tf32 or 16 f16)
                    const uint64_t ko = (uint64_t)(k * 32 >> 4);
                    if (F16) {
                        mma_f16(d, ah + ko, bh + ko, (kc > 0 || k > 0) ? 1u : 0u);
                        mma_f16(d, ah + ko, bl + ko, 1u);
                        mma_f16(d, al + ko, bh + ko, 1u);
                    } else {
                        mma_tf32(d, ah + ko, bh + ko, (kc > 0 || k > 0) ? 1u : 0u);
                        mma_tf32(d, ah + ko, bl + ko, 1u);
                        mma_tf32(d, al + ko, bh + ko, 1u);
                    }
                }
                mma_commit(empty_bar + 8 * s);
                if (kc == nkc - 1) mma_commit(accf_bar + 8 * acc);
            }
        }
        __syncwarp();
    } else if (warp >= 4) {
        // ---------------- drainers ----------------
        const int dw = warp - 4;                        // 0..7
        const int quad = warp & 3;                      // TMEM lane quadrant of this warp
        const int half = dw >> 2;                       // which 64 columns
        double acc64[64];
#pragma unroll
        for (int j = 0; j < 64; ++j) acc64[j] = 0.0;
        bool ok = true;
        for (int gi = 0; gi < ng && ok; ++gi) {
            const int acc = gi & 1;
            // f16 form: the product of this thread's operator-row scale and
            // each column's source-row scale (lane l holds columns l and
            // 32 + l of this warp's 64; shuffled out below); empty slots 0
            float rs = 1.0f, cs0 = 0.0f, cs1 = 0.0f;
            if (F16) {
                const int g = g0 + gi;
                const int32_t *gs = a.group_sources + (int64_t)g * TC_TW + half * 64;
                const int32_t s0 = gs[lane], s1 = gs[32 + lane];
                cs0 = s0 >= 0 ? a.src_rinv[s0 - a.src_row_base] : 0.0f;
                cs1 = s1 >= 0 ? a.src_rinv[s1 - a.src_row_base] : 0.0f;
                rs = a.mat_rinv[(int64_t)a.group_class[g] * a.rows_pad + row0 + quad * 32 + lane];
            }
            ok = mbar_wait_or_abort(accf_bar + 8 * acc, (gi >> 1) & 1, abort_flag, a.wait_cycles);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            tc_fence_after();
            const uint32_t taddr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(acc * TC_TW + half * 64);
#pragma unroll
            for (int c0 = 0; c0 < 64; c0 += 16) {
                uint32_t r[16];
                tmem_ld16(taddr + c0, r);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    if (F16) {
                        // powers of two, applied in two FP32 products (column
                        // scale first): exact whenever the contribution lies
                        // in the FP32 normal range, the range the mixed form's
                        // FP32 near field needs anyway
                        // (an empty slot's scale is 0, the same in every lane
                        // of the warp: the whole warp skips that column)
                        const int col = c0 + j;
                        const float cs = __shfl_sync(0xffffffffu, col < 32 ? cs0 : cs1, col & 31);
                        if (cs != 0.0f)
                            acc64[col] += (double)((__uint_as_float(r[j]) * cs) * rs);
                    } else {
                        acc64[c0 + j] += (double)__uint_as_float(r[j]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acce_bar + 8 * acc);
        }
        if (ok && ng > 0) {
            const int row = row0 + quad * 32 + lane;
            const double scale = a.tile_scale[tile];
            if (row < a.n) {
#pragma unroll
                for (int j = 0; j < 64; ++j) {
                    const int32_t t = a.tile_targets[(int64_t)tile * TC_TW + half * 64 + j];
                    if (t >= 0) atomicAdd(a.tgt + (int64_t)(t - a.tbase) * a.n + row, scale * acc64[j]);
                }
            }
        }
    }

    if (threadIdx.x == 0 && *abort_flag && a.status) atomicExch(a.status, ST_TIMEOUT_MMA);
    tc_fence_before();
    __syncthreads();
    if (*abort_flag) {
        // let copies and tensor-core work still in flight finish before the
        // shared and tensor memory are released
        const long long t0 = clock64();
        while (clock64() - t0 < 20000000) {}
    }
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS)
                     : "memory");
    }
}

__device__ __forceinline__ float tf32_rna(float x)
{
    uint32_t u;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(u) : "f"(x));
    return __uint_as_float(u);
}

__global__ void split_tf32x2_kernel(int64_t nmat, int rows, int cols, const double *__restrict__ in,
                                    int rows_pad, int cols_pad, float *__restrict__ hi,
                                    float *__restrict__ lo)
{
    const int64_t total = nmat * rows_pad * cols_pad;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % cols_pad);
        const int64_t mr = e / cols_pad;
        const int r = (int)(mr % rows_pad);
        const int64_t m = mr / rows_pad;
        const double v = (r < rows && c < cols) ? in[(m * rows + r) * cols + c] : 0.0;
        const float h = tf32_rna((float)v);
        hi[e] = h;
        lo[e] = tf32_rna((float)(v - (double)h));
    }
}

// f16 hi/lo planes with a power-of-two scale per row: one warp per padded
// row. Row r of matrix m is scaled by 2^e with e chosen so that the row's
// largest magnitude lands in [2^13, 2^14) (|e| <= 126), then split as
// hi = f16(x 2^e), lo = f16(x 2^e - hi); inv[row] = 2^-e. Zero rows and
// padding rows get hi = lo = 0 and inv = 1. The scaling keeps every row in
// the f16 exponent range whatever the magnitudes of the data.
__global__ void split_f16x2_rowscale_kernel(int64_t nrows_total, int rows, int cols,
                                            const double *__restrict__ in, int rows_pad,
                                            int cols_pad, __half *__restrict__ hi,
                                            __half *__restrict__ lo, float *__restrict__ inv)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t wr = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); wr < nrows_total;
         wr += warps) {
        const int r = (int)(wr % rows_pad);
        const int64_t m = wr / rows_pad;
        const bool real_row = r < rows;
        const double *row = in + (m * rows + r) * (int64_t)cols;
        double mx = 0.0;
        if (real_row)
            for (int c = lane; c < cols; c += 32) mx = fmax(mx, fabs(row[c]));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        int e = 0;
        if (mx > 0.0) {
            int ex;
            frexp(mx, &ex);              // mx = f 2^ex, f in [0.5, 1)
            e = 14 - ex;                 // mx 2^e in [2^13, 2^14)
            e = e > 126 ? 126 : (e < -126 ? -126 : e);
        }
        __half *h = hi + wr * cols_pad;
        __half *l = lo + wr * cols_pad;
        for (int c = lane; c < cols_pad; c += 32) {
            const double v = (real_row && c < cols) ? ldexp(row[c], e) : 0.0;
            const __half vh = __double2half(v);
            h[c] = vh;
            l[c] = __double2half(v - (double)__half2float(vh));
        }
        if (lane == 0) inv[wr] = ldexpf(1.0f, -e);
    }
}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_split_f16x2_rowscale(int64_t nmat, int32_t rows, int32_t cols, const double *in,
                               int32_t rows_pad, int32_t cols_pad, void *hi, void *lo,
                               float *row_inv, void *stream)
{
    if (nmat < 0 || rows < 0 || cols < 0 || rows_pad < rows || cols_pad < cols)
        return bad_arg("split_f16x2_rowscale: bad sizes");
    if (nmat == 0 || rows_pad == 0 || cols_pad == 0) return SUMPY_OK;
    if ((rows > 0 && cols > 0 && !in) || !hi || !lo || !row_inv)
        return bad_arg("split_f16x2_rowscale: null pointer");
    const int64_t nr = nmat * rows_pad;
    const int64_t blocks = std::min<int64_t>((nr + 7) / 8, 148 * 16);
    split_f16x2_rowscale_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(
        nr, rows, cols, in, rows_pad, cols_pad, static_cast<__half *>(hi),
        static_cast<__half *>(lo), row_inv);
    return check_launch("split_f16x2_rowscale_kernel");
}

int sumpy_split_tf32x2(int64_t nmat, int32_t rows, int32_t cols, const double *in,
                       int32_t rows_pad, int32_t cols_pad, float *hi, float *lo, void *stream)
{
    if (nmat < 0 || rows < 0 || cols < 0 || rows_pad < rows || cols_pad < cols)
        return bad_arg("split_tf32x2: bad sizes");
    if (nmat == 0 || rows_pad == 0 || cols_pad == 0) return SUMPY_OK;
    if ((rows > 0 && cols > 0 && !in) || !hi || !lo) return bad_arg("split_tf32x2: null pointer");
    const int64_t total = nmat * rows_pad * cols_pad;
    const int64_t blocks = std::min<int64_t>((total + 255) / 256, 148 * 16);
    split_tf32x2_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(nmat, rows, cols, in, rows_pad,
                                                                        cols_pad, hi, lo);
    return check_launch("split_tf32x2_kernel");
}

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                    const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                    const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// fp32 or f16 tensor map over [dims[rank-1]]...[dims[0]], ROWB-byte swizzle,
// box {one ROWB-byte row of K, box1, 1}
static bool make_map(CUtensorMap *m, const void *ptr, bool f16, int rank, const uint64_t *dims,
                     uint32_t box1)
{
    EncodeTiledFn fn = encode_tiled_fn();
    if (!fn) return false;
    const uint64_t es = f16 ? 2 : 4;
    cuuint64_t gdim[3], gstride[2];
    cuuint32_t box[3] = {(cuuint32_t)(ROWB / es), box1, 1}, estr[3] = {1, 1, 1};
    for (int i = 0; i < rank; ++i) gdim[i] = dims[i];
    gstride[0] = dims[0] * es;
    if (rank == 3) gstride[1] = dims[0] * dims[1] * es;
    CUresult r = fn(m, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank,
                    const_cast<void *>(ptr), gdim, gstride,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    ROWB == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // extern "C"

// n = real coefficients per expansion row: ncoeff for real data, 2 ncoeff for
// complex data stored as interleaved (re, im) with the real embedding of the
// complex operators. f16: operand planes are f16 with the row scales
// mats_rinv [nclasses][rows_pad] and src_rinv [src_nrows]; otherwise fp32
// holding tf32 values (the row-scale pointers are ignored).
static int m2l_tc_launch(
    bool f16, int n, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const void *mats_hi, const void *mats_lo, const float *mats_rinv,
    int32_t rows_pad, int32_t k_pad, int32_t src_nrows, int32_t src_base_ibox,
    const void *src_hi, const void *src_lo, const float *src_rinv, int32_t tgt_base_ibox,
    double *tgt_expansions, int32_t *status, void *stream, int32_t k_split = 1)
{
    const char *who = f16 ? "m2l_f16x3" : "m2l_tf32x3";
    const int kc = f16 ? ROWB / 2 : ROWB / 4;   // K per stage
    if (tile_width != TC_TW) return bad_arg((std::string(who) + ": tile_width must be 128").c_str());
    if (k_pad < n || k_pad % kc)
        return bad_arg((std::string(who) + ": k_pad must be a multiple of " + std::to_string(kc) +
                       " >= ncoeff").c_str());
    if (k_split < 1 || k_split > k_pad / kc)
        return bad_arg((std::string(who) + ": k_split must be in [1, k_pad / " +
                       std::to_string(kc) + "]").c_str());
    if (rows_pad < n || rows_pad % TC_M)
        return bad_arg((std::string(who) + ": rows_pad must be a multiple of 128 >= ncoeff").c_str());
    if (nitems < 0 || nclasses <= 0 || src_nrows < 1)
        return bad_arg((std::string(who) + ": bad sizes").c_str());
    if (nitems == 0) return SUMPY_OK;
    if (!item_tile || !item_group_begin || !item_group_end || !tile_targets || !tile_scale ||
        !group_class || !group_sources || !mats_hi || !mats_lo || !src_hi || !src_lo ||
        !tgt_expansions || (f16 && (!mats_rinv || !src_rinv)))
        return bad_arg((std::string(who) + ": null pointer argument").c_str());
    if ((reinterpret_cast<uintptr_t>(mats_hi) | reinterpret_cast<uintptr_t>(mats_lo) |
         reinterpret_cast<uintptr_t>(src_hi) | reinterpret_cast<uintptr_t>(src_lo)) & 15)
        return bad_arg((std::string(who) + ": operand planes must be 16-byte aligned").c_str());
    // set on every launch (a cheap host call): an attribute remembered per
    // device would be lost with a context that was torn down and recreated
    cudaError_t e = f16 ? cudaFuncSetAttribute(m2l_tc_kernel<true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM)
                        : cudaFuncSetAttribute(m2l_tc_kernel<false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    if (e != cudaSuccess) {
        set_last_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        return SUMPY_ELAUNCH;
    }
    CUtensorMap ma_hi, ma_lo, mb_hi, mb_lo;
    const uint64_t adims[3] = {(uint64_t)k_pad, (uint64_t)rows_pad, (uint64_t)nclasses};
    const uint64_t bdims[2] = {(uint64_t)k_pad, (uint64_t)src_nrows};
    // one 128-row block of operator rows: the TMA box stops at the last real
    // row (the MMA's rows past it hold stale shared memory and are never
    // stored); several blocks: whole 128-row boxes of the zero-padded planes
    const int32_t a_rows = rows_pad == TC_M ? n : TC_M;
    if (!make_map(&ma_hi, mats_hi, f16, 3, adims, (uint32_t)a_rows) ||
        !make_map(&ma_lo, mats_lo, f16, 3, adims, (uint32_t)a_rows) ||
        !make_map(&mb_hi, src_hi, f16, 2, bdims, 1) || !make_map(&mb_lo, src_lo, f16, 2, bdims, 1)) {
        set_last_error(std::string(who) + ": tensor map encoding failed");
        return SUMPY_EINVAL;
    }
    TcArgs a;
    a.n = n; a.k_pad = k_pad;
    a.item_tile = item_tile; a.item_g0 = item_group_begin; a.item_g1 = item_group_end;
    a.tile_targets = tile_targets; a.tile_scale = tile_scale;
    a.group_class = group_class; a.group_sources = group_sources;
    a.src_hi = src_hi; a.src_lo = src_lo;
    a.src_rinv = src_rinv; a.mat_rinv = mats_rinv; a.rows_pad = rows_pad; a.a_rows = a_rows;
    a.src_row_base = src_base_ibox; a.zero_row = src_nrows - 1;
    a.tbase = tgt_base_ibox; a.tgt = tgt_expansions; a.status = status;
    a.wait_cycles = wait_cycles_budget();
    dim3 grid(nitems, rows_pad / TC_M, k_split);
    if (f16)
        m2l_tc_kernel<true><<<grid, TC_THREADS, TC_SMEM, as_stream(stream)>>>(a, ma_hi, ma_lo,
                                                                             mb_hi, mb_lo);
    else
        m2l_tc_kernel<false><<<grid, TC_THREADS, TC_SMEM, as_stream(stream)>>>(a, ma_hi, ma_lo,
                                                                              mb_hi, mb_lo);
    return check_launch(f16 ? "m2l_tc_kernel<f16>" : "m2l_tc_kernel<tf32>");
}

static int m2l_tf32x3_launch(
    int n, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const float *mats_hi, const float *mats_lo, int32_t rows_pad, int32_t k_pad,
    int32_t src_nrows, int32_t src_base_ibox, const float *src_hi, const float *src_lo,
    int32_t tgt_base_ibox, double *tgt_expansions, int32_t *status, void *stream,
    int32_t k_split = 1)
{
    return m2l_tc_launch(false, n, nitems, item_tile, item_group_begin, item_group_end,
                         tile_width, tile_targets, tile_scale, group_class, group_sources,
                         nclasses, mats_hi, mats_lo, nullptr, rows_pad, k_pad, src_nrows,
                         src_base_ibox, src_hi, src_lo, nullptr, tgt_base_ibox, tgt_expansions,
                         status, stream, k_split);
}

extern "C" {

int sumpy_m2l_translation_classes_tf32x3(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const float *mats_hi, const float *mats_lo, int32_t rows_pad, int32_t k_pad,
    int32_t src_nrows, int32_t src_base_ibox, const float *src_hi, const float *src_lo,
    int32_t tgt_base_ibox, double *tgt_expansions, int32_t *status, void *stream)
{
    if (order < 0 || order > SUMPY_MAX_ORDER) {
        set_last_error("m2l_tf32x3: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    return m2l_tf32x3_launch(ncoeff_of(order), nitems, item_tile, item_group_begin,
                             item_group_end, tile_width, tile_targets, tile_scale, group_class,
                             group_sources, nclasses, mats_hi, mats_lo, rows_pad, k_pad,
                             src_nrows, src_base_ibox, src_hi, src_lo, tgt_base_ibox,
                             tgt_expansions, status, stream);
}

int sumpy_class_gemm_tf32x3(
    int32_t n, int32_t k_split, int32_t nitems, const int32_t *item_tile,
    const int32_t *item_group_begin, const int32_t *item_group_end, int32_t tile_width,
    const int32_t *tile_targets, const double *tile_scale, const int32_t *group_class,
    const int32_t *group_sources, int32_t nclasses, const float *mats_hi, const float *mats_lo,
    int32_t rows_pad, int32_t k_pad, int32_t src_nrows, int32_t src_base_ibox,
    const float *src_hi, const float *src_lo, int32_t tgt_base_ibox, double *tgt_expansions,
    int32_t *status, void *stream)
{
    if (n < 1 || n > 2 * ncoeff_of(SUMPY_MAX_ORDER)) return bad_arg("class gemm tf32x3: bad n");
    return m2l_tf32x3_launch(n, nitems, item_tile, item_group_begin, item_group_end, tile_width,
                             tile_targets, tile_scale, group_class, group_sources, nclasses,
                             mats_hi, mats_lo, rows_pad, k_pad, src_nrows, src_base_ibox, src_hi,
                             src_lo, tgt_base_ibox, tgt_expansions, status, stream, k_split);
}

int sumpy_helmholtz_m2l_translation_classes_tf32x3(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const float *mats_hi, const float *mats_lo, int32_t rows_pad, int32_t k_pad,
    int32_t src_nrows, int32_t src_base_ibox, const float *src_hi, const float *src_lo,
    int32_t tgt_base_ibox, double *tgt_expansions, int32_t *status, void *stream)
{
    if (order < 0 || order > SUMPY_MAX_ORDER) {
        set_last_error("helmholtz m2l_tf32x3: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    return m2l_tf32x3_launch(2 * ncoeff_of(order), nitems, item_tile, item_group_begin,
                             item_group_end, tile_width, tile_targets, tile_scale, group_class,
                             group_sources, nclasses, mats_hi, mats_lo, rows_pad, k_pad,
                             src_nrows, src_base_ibox, src_hi, src_lo, tgt_base_ibox,
                             tgt_expansions, status, stream);
}

int sumpy_m2l_translation_classes_f16x3(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const void *mats_hi, const void *mats_lo, const float *mats_rinv,
    int32_t rows_pad, int32_t k_pad, int32_t src_nrows, int32_t src_base_ibox,
    const void *src_hi, const void *src_lo, const float *src_rinv, int32_t tgt_base_ibox,
    double *tgt_expansions, int32_t *status, void *stream)
{
    if (order < 0 || order > SUMPY_MAX_ORDER) {
        set_last_error("m2l_f16x3: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    return m2l_tc_launch(true, ncoeff_of(order), nitems, item_tile, item_group_begin,
                         item_group_end, tile_width, tile_targets, tile_scale, group_class,
                         group_sources, nclasses, mats_hi, mats_lo, mats_rinv, rows_pad, k_pad,
                         src_nrows, src_base_ibox, src_hi, src_lo, src_rinv, tgt_base_ibox,
                         tgt_expansions, status, stream);
}

int sumpy_helmholtz_m2l_translation_classes_f16x3(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const void *mats_hi, const void *mats_lo, const float *mats_rinv,
    int32_t rows_pad, int32_t k_pad, int32_t src_nrows, int32_t src_base_ibox,
    const void *src_hi, const void *src_lo, const float *src_rinv, int32_t tgt_base_ibox,
    double *tgt_expansions, int32_t *status, void *stream)
{
    if (order < 0 || order > SUMPY_MAX_ORDER) {
        set_last_error("helmholtz m2l_f16x3: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    return m2l_tc_launch(true, 2 * ncoeff_of(order), nitems, item_tile, item_group_begin,
                         item_group_end, tile_width, tile_targets, tile_scale, group_class,
                         group_sources, nclasses, mats_hi, mats_lo, mats_rinv, rows_pad, k_pad,
                         src_nrows, src_base_ibox, src_hi, src_lo, src_rinv, tgt_base_ibox,
                         tgt_expansions, status, stream);
}

int sumpy_class_gemm_f16x3(
    int32_t n, int32_t k_split, int32_t nitems, const int32_t *item_tile,
    const int32_t *item_group_begin, const int32_t *item_group_end, int32_t tile_width,
    const int32_t *tile_targets, const double *tile_scale, const int32_t *group_class,
    const int32_t *group_sources, int32_t nclasses, const void *mats_hi, const void *mats_lo,
    const float *mats_rinv, int32_t rows_pad, int32_t k_pad, int32_t src_nrows,
    int32_t src_base_ibox, const void *src_hi, const void *src_lo, const float *src_rinv,
    int32_t tgt_base_ibox, double *tgt_expansions, int32_t *status, void *stream)
{
    if (n < 1 || n > 2 * ncoeff_of(SUMPY_MAX_ORDER)) return bad_arg("class gemm f16x3: bad n");
    return m2l_tc_launch(true, n, nitems, item_tile, item_group_begin, item_group_end,
                         tile_width, tile_targets, tile_scale, group_class, group_sources,
                         nclasses, mats_hi, mats_lo, mats_rinv, rows_pad, k_pad, src_nrows,
                         src_base_ibox, src_hi, src_lo, src_rinv, tgt_base_ibox, tgt_expansions,
                         status, stream, k_split);
}

// ---------------------------------------------------------------------------
// Variant of the tensor-core M2L that allocates nothing.
//
// Some callers cannot allocate device memory once they are running: host
// applications that fix their device-memory budget at start-up (a solver
// framework owning one pool for everything, a real-time or certified loop
// that forbids allocation after initialisation), or code embedded where an
// allocation would synchronise the device. This entry point keeps the TF32
// planes of the source multipoles -- the only scratch the tensor-core M2L
// needs -- in a file-scope device array instead of caller memory.
//
// Limits: (nsrc_boxes + 1) * k_pad <= NOALLOC_ROWS * NOALLOC_KPAD floats per
// plane, i.e. 8,191 source boxes at k_pad = 128 (orders <= 10); larger
// requests are rejected. Every GPU that loads this library's module holds
// the array (8 MiB) until the process exits; with CUDA's default lazy module
// loading the module, and with it the array, is loaded by the first call
// into this file's kernels on that device (this entry point or the regular
// tensor-core M2L), so a caller with a fixed budget makes one such call
// while it initialises (or sets CUDA_MODULE_LOADING=EAGER) and makes it
// before any stream capture. All calls share the array and it keeps the
// previous call's contents; the zero row the kernel needs is cleared on
// every call. Calls that overlap on the GPU (different streams, or another
// thread) race on the array and must be serialised by the caller.
constexpr int64_t NOALLOC_ROWS = 8192;
constexpr int64_t NOALLOC_KPAD = 128;
static __device__ __align__(256) float g_noalloc_planes[2 * NOALLOC_ROWS * NOALLOC_KPAD];

// Device address of g_noalloc_planes in the current device's context. Host
// code cannot use the symbol's name as a device address, so every call looks
// the address up (it allocates nothing once the module is loaded); nothing is
// cached, so a context that was torn down and created again is never used
// through a stale address.
static float *noalloc_planes()
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_planes);
    if (e != cudaSuccess) {
        set_last_error(std::string("m2l_tf32x3_noalloc: cudaGetSymbolAddress: ") +
                       cudaGetErrorString(e));
        return nullptr;
    }
    return static_cast<float *>(p);
}

int sumpy_m2l_translation_classes_tf32x3_noalloc(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const float *mats_hi, const float *mats_lo, int32_t rows_pad, int32_t k_pad,
    int32_t nsrc_boxes, int32_t src_base_ibox, const double *src_expansions,
    int32_t tgt_base_ibox, double *tgt_expansions, int32_t *status, void *stream)
{
    if (order < 0 || order > SUMPY_MAX_ORDER) {
        set_last_error("m2l_tf32x3_noalloc: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    const int n = ncoeff_of(order);
    if (nsrc_boxes < 0 || k_pad < n || k_pad % 32) return bad_arg("m2l_tf32x3_noalloc: bad sizes");
    if (k_pad > NOALLOC_KPAD || (int64_t)(nsrc_boxes + 1) * k_pad > NOALLOC_ROWS * NOALLOC_KPAD) {
        set_last_error("m2l_tf32x3_noalloc: request exceeds the built-in scratch: needs (nsrc_boxes+1)*k_pad <= " +
                       std::to_string(NOALLOC_ROWS * NOALLOC_KPAD) + " and k_pad <= " +
                       std::to_string(NOALLOC_KPAD) + " (got nsrc_boxes=" +
                       std::to_string(nsrc_boxes) + ", k_pad=" + std::to_string(k_pad) + ")");
        return SUMPY_EINVAL;
    }
    if (nsrc_boxes > 0 && !src_expansions) return bad_arg("m2l_tf32x3_noalloc: null pointer argument");
    float *hi = noalloc_planes();
    if (!hi) return SUMPY_ELAUNCH;
    float *lo = hi + NOALLOC_ROWS * NOALLOC_KPAD;
    cudaStream_t st = as_stream(stream);
    const size_t zero_off = (size_t)nsrc_boxes * k_pad;
    if (cudaMemsetAsync(hi + zero_off, 0, sizeof(float) * k_pad, st) != cudaSuccess ||
        cudaMemsetAsync(lo + zero_off, 0, sizeof(float) * k_pad, st) != cudaSuccess)
        return check_launch("m2l_tf32x3_noalloc: clearing the zero row");
    int rc = sumpy_split_tf32x2(nsrc_boxes, 1, n, src_expansions, 1, k_pad, hi, lo, stream);
    if (rc) return rc;
    return sumpy_m2l_translation_classes_tf32x3(
        order, nitems, item_tile, item_group_begin, item_group_end, tile_width, tile_targets,
        tile_scale, group_class, group_sources, nclasses, mats_hi, mats_lo, rows_pad, k_pad,
        nsrc_boxes + 1, src_base_ibox, hi, lo, tgt_base_ibox, tgt_expansions, status, stream);
}

}  // extern "C"
