// M2L per translation class as dense GEMMs (FP64).
//
// sumpy applies M2L per target box and List-2 source with the translation
// class's derivative vector, via FFT or a Toeplitz product
// (sumpy/e2e.py:310-558, sumpy/expansion/m2l.py:363-389, 913-1001). In exact
// arithmetic each class c is the linear map
//     L[t] += (r_tgt/r_src)^|t| sum_s M[s] D_c[s+t]
// so with T_c[t][s] (one n x n matrix per class, built on the host) the
// M2L of a level is sum_c T_c * M[:, sources of class c].
//
// Schedule (same form as the tensor-core kernel): tiles of 64 target boxes
// with one scale each (the level's operator factor), per tile the class
// groups (one source box per target slot, -1 = none), and work items = up
// to G consecutive groups of one tile; all levels in one launch. A CTA runs
// one work item for ROWS (64 or 128) output rows: C += T_c * B_g over the
// item's groups, the accumulator in registers, added to the local
// expansions with FP64 atomics at the end (items of one tile may overlap in
// time). Thread (ty, tx) owns rows ty + (ROWS/8) r and target slots
// tx + 8 c (r, c < 8): each shared-memory read of a k-step is conflict-free.
// The next k-chunk of both operands is fetched into registers while the
// current one is multiplied.
#include <algorithm>

#include "common.cuh"

namespace sumpy {
namespace {

constexpr int TW = 64;  // target boxes per tile
constexpr int KC = 8;   // k-chunk

template <int ROWS>
struct Chunk {
    static constexpr int NT = ROWS;
    static constexpr int A_PER = ROWS * KC / NT;  // = KC
    static constexpr int B_PER = TW * KC / NT;
    double a[A_PER];
    double b[B_PER];
};

// CG: read the source expansions through L2 only (ld.global.cg) -- needed
// when other CTAs of the same launch wrote them (the level-chained kernel)
template <int ROWS, bool CG = false>
__device__ __forceinline__ void fetch(Chunk<ROWS> &ch, const double *__restrict__ A,
                                      const double *__restrict__ src, const int32_t *srcs, int n,
                                      int row0, int k0, int32_t sbase)
{
    constexpr int NT = ROWS;
#pragma unroll
    for (int u = 0; u < Chunk<ROWS>::A_PER; ++u) {
        const int idx = threadIdx.x + u * NT;
        const int r = idx / KC, kk = idx % KC;
        const int row = row0 + r, k = k0 + kk;
        ch.a[u] = (row < n && k < n) ? A[(int64_t)row * n + k] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < Chunk<ROWS>::B_PER; ++u) {
        const int idx = threadIdx.x + u * NT;
        const int slot = idx / KC, kk = idx % KC;
        const int32_t s = srcs[slot];
        const int k = k0 + kk;
        const double *p = src + (int64_t)(s - sbase) * n + k;
        ch.b[u] = (s >= 0 && k < n) ? (CG ? __ldcg(p) : *p) : 0.0;
    }
}

// One work item (a range of class groups of one tile) for output rows
// [row0, row0 + ROWS) and k-chunks [kcb, kcb + nkc): C += T_c * B_g over the
// item's groups, accumulated in registers and added to the local expansions
// with FP64 atomics (items of one tile may overlap in time). Thread (ty, tx)
// owns rows ty + (ROWS/8) r and target slots tx + 8 c (r, c < 8): each
// shared-memory read of a k-step is conflict-free. The next k-chunk of both
// operands is fetched into registers while the current one is multiplied.
template <int ROWS, bool CG>
__device__ __forceinline__ void class_gemm_item(
    int n, int item, int row0, int kcb, int nkc, const int32_t *__restrict__ item_tile,
    const int32_t *__restrict__ item_g0, const int32_t *__restrict__ item_g1,
    const int32_t *__restrict__ tile_targets, const double *__restrict__ tile_scale,
    const int32_t *__restrict__ group_class, const int32_t *__restrict__ group_sources,
    const double *__restrict__ mats, int32_t sbase, const double *__restrict__ src,
    int32_t tbase, double *__restrict__ tgt)
{
    constexpr int NT = ROWS;          // (ROWS / 8) x 8 threads
    constexpr int RG = ROWS / 8;      // row groups
    __shared__ double As[2][KC][ROWS + 1];
    __shared__ double Bs[2][KC][TW + 1];
    __shared__ int32_t srcs[2][TW];

    const int tile = item_tile[item];
    const int g0 = item_g0[item], g1 = item_g1[item];
    const int tid = threadIdx.x;
    const int tx = tid % 8, ty = tid / 8;
    const int total = (g1 - g0) * nkc;
    if (total <= 0) return;

    double acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;

    auto load_srcs = [&](int g, int buf) {
        for (int s = tid; s < TW; s += NT) srcs[buf][s] = group_sources[(int64_t)g * TW + s];
    };
    auto store = [&](const Chunk<ROWS> &ch, int buf) {
#pragma unroll
        for (int u = 0; u < Chunk<ROWS>::A_PER; ++u) {
            const int idx = tid + u * NT;
            As[buf][idx % KC][idx / KC] = ch.a[u];
        }
#pragma unroll
        for (int u = 0; u < Chunk<ROWS>::B_PER; ++u) {
            const int idx = tid + u * NT;
            Bs[buf][idx % KC][idx / KC] = ch.b[u];
        }
    };

    Chunk<ROWS> ch;
    load_srcs(g0, 0);
    __syncthreads();
    fetch<ROWS, CG>(ch, mats + (int64_t)group_class[g0] * n * n, src, srcs[0], n, row0,
                    kcb * KC, sbase);
    store(ch, 0);
    __syncthreads();
    for (int it = 0; it < total; ++it) {
        const int buf = it & 1;
        const int nxt = it + 1;
        if (nxt < total) {
            const int g = g0 + nxt / nkc, kc = nxt % nkc;
            const int sb = (g - g0) & 1;
            if (kc == 0) {
                load_srcs(g, sb);
                __syncthreads();
            }
            fetch<ROWS, CG>(ch, mats + (int64_t)group_class[g] * n * n, src, srcs[sb], n, row0,
                            (kcb + kc) * KC, sbase);
        }
#pragma unroll 4
        for (int kk = 0; kk < KC; ++kk) {
            double a[8], b[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) a[r] = As[buf][kk][ty + RG * r];
#pragma unroll
            for (int c = 0; c < 8; ++c) b[c] = Bs[buf][kk][tx + 8 * c];
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
        }
        if (nxt < total) store(ch, buf ^ 1);
        __syncthreads();
    }
    const double scale = tile_scale[tile];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int32_t t = tile_targets[(int64_t)tile * TW + tx + 8 * c];
        if (t < 0) continue;
        double *o = tgt + (int64_t)(t - tbase) * n;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int row = row0 + ty + RG * r;
            if (row < n) atomicAdd(o + row, scale * acc[r][c]);
        }
    }
}

template <int ROWS>
__global__ void __launch_bounds__(ROWS)
m2l_f64_kernel(int n, const int32_t *__restrict__ item_tile, const int32_t *__restrict__ item_g0,
               const int32_t *__restrict__ item_g1, const int32_t *__restrict__ tile_targets,
               const double *__restrict__ tile_scale, const int32_t *__restrict__ group_class,
               const int32_t *__restrict__ group_sources, const double *__restrict__ mats,
               int32_t sbase, const double *__restrict__ src, int32_t tbase,
               double *__restrict__ tgt)
{
    // split K: CTA z of gridDim.z takes k-chunks [kcb, kcb + nkc) (all when 1)
    const int nkc_all = (n + KC - 1) / KC;
    const int kcb = (int)((int64_t)blockIdx.z * nkc_all / gridDim.z);
    const int nkc = (int)((int64_t)(blockIdx.z + 1) * nkc_all / gridDim.z) - kcb;
    class_gemm_item<ROWS, false>(n, blockIdx.x, blockIdx.y * ROWS, kcb, nkc, item_tile, item_g0,
                                 item_g1, tile_targets, tile_scale, group_class, group_sources,
                                 mats, sbase, src, tbase, tgt);
}

// Level-chained form for M2M / L2L: the GEMMs of all levels in one
// persistent launch. Work units (item, row block, k-chunk range) of all
// levels are numbered level after level in the order the chain runs (M2M:
// finest parents first; L2L: coarsest children first) and handed out by an
// atomic counter; a unit of chain step L starts once every unit of step L - 1
// has finished (a per-step done counter), because its sources are that
// step's targets. Units are dispatched in order only to running CTAs, so the
// units a waiting CTA depends on are held by running CTAs: no deadlock, with
// or without co-residency. Each wait is bounded (the process-wide wait
// budget); a wait that runs out writes status 2 and stops the CTA.
// Expansions of every level live in one flat [nboxes][n] array (box ids are
// rows); sources written earlier in the launch are read through L2.
struct ChainArgs {
    int n, nsteps;
    const int32_t *step_unit_start;    // [nsteps + 1] first unit of each step
    const int32_t *step_item_start;    // [nsteps] first item of each step
    const int32_t *step_ksplit;        // [nsteps]
    int32_t nrowblk;
    const int32_t *item_tile, *item_g0, *item_g1, *tile_targets;
    const double *tile_scale;
    const int32_t *group_class, *group_sources;
    const double *mats;
    double *expansions;
    int32_t *queue;                    // [0] next unit, [1 + L] units of step L done
    int32_t *status;
    long long wait_cycles;
};

constexpr int CHAIN_MAX_STEPS = 64;

template <int ROWS>
__global__ void __launch_bounds__(ROWS)
class_gemm_chain_kernel(ChainArgs a)
{
    __shared__ int32_t s_unit_start[CHAIN_MAX_STEPS + 1];
    __shared__ int s_unit, s_stop;
    for (int i = threadIdx.x; i <= a.nsteps; i += blockDim.x) s_unit_start[i] = a.step_unit_start[i];
    __syncthreads();
    const int total = s_unit_start[a.nsteps];
    const int nkc_all = (a.n + KC - 1) / KC;
    while (true) {
        if (threadIdx.x == 0) {
            s_unit = atomicAdd(a.queue, 1);
            s_stop = 0;
        }
        __syncthreads();
        const int u = s_unit;
        if (u >= total) break;
        int L = 0;
        while (L + 1 < a.nsteps && s_unit_start[L + 1] <= u) ++L;
        if (threadIdx.x == 0 && L > 0) {
            const int need = s_unit_start[L] - s_unit_start[L - 1];
            const long long t0 = clock64();
            while (*reinterpret_cast<volatile int32_t *>(a.queue + L) < need) {
                if (clock64() - t0 > a.wait_cycles) {
                    s_stop = 1;
                    if (a.status) atomicExch(a.status, 2);
                    break;
                }
            }
            __threadfence();
        }
        __syncthreads();
        if (s_stop) break;
        const int ks = a.step_ksplit[L];
        const int local = u - s_unit_start[L];
        const int per_item = a.nrowblk * ks;
        const int item = a.step_item_start[L] + local / per_item;
        const int rem = local % per_item;
        const int y = rem / ks, z = rem % ks;
        const int kcb = (int)((int64_t)z * nkc_all / ks);
        const int nkc = (int)((int64_t)(z + 1) * nkc_all / ks) - kcb;
        class_gemm_item<ROWS, true>(a.n, item, y * ROWS, kcb, nkc, a.item_tile, a.item_g0,
                                    a.item_g1, a.tile_targets, a.tile_scale, a.group_class,
                                    a.group_sources, a.mats, 0, a.expansions, 0, a.expansions);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(a.queue + 1 + L, 1);
    }
}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

// n = real coefficients per expansion row (ncoeff, or 2 ncoeff for complex
// data as interleaved (re, im) with real-embedded operators).
static int m2l_f64_launch(
    int n, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const double *class_matrices, int32_t src_base_ibox,
    const double *src_expansions, int32_t tgt_base_ibox, double *tgt_expansions, void *stream,
    int32_t k_split = 1)
{
    if (tile_width != TW) return bad_arg("m2l: tile_width must be 64");
    if (n < 1 || k_split < 1 || k_split > (n + KC - 1) / KC)
        return bad_arg("m2l: k_split must be in [1, number of 8-wide k-chunks]");
    if (nitems < 0 || nclasses < 0) return bad_arg("m2l: negative size");
    if (nitems == 0) return SUMPY_OK;
    if (!item_tile || !item_group_begin || !item_group_end || !tile_targets || !tile_scale ||
        !group_class || !group_sources || !class_matrices || !src_expansions || !tgt_expansions)
        return bad_arg("m2l: null pointer argument");
    cudaStream_t st = as_stream(stream);
    if (n <= 64) {
        dim3 grid(nitems, 1, k_split);
        m2l_f64_kernel<64><<<grid, 64, 0, st>>>(n, item_tile, item_group_begin, item_group_end,
                                                tile_targets, tile_scale, group_class,
                                                group_sources, class_matrices, src_base_ibox,
                                                src_expansions, tgt_base_ibox, tgt_expansions);
    } else {
        dim3 grid(nitems, (n + 127) / 128, k_split);
        m2l_f64_kernel<128><<<grid, 128, 0, st>>>(n, item_tile, item_group_begin, item_group_end,
                                                  tile_targets, tile_scale, group_class,
                                                  group_sources, class_matrices, src_base_ibox,
                                                  src_expansions, tgt_base_ibox, tgt_expansions);
    }
    return check_launch("m2l_f64_kernel");
}

extern "C" {

int sumpy_m2l_translation_classes_f64(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const double *class_matrices, int32_t src_base_ibox,
    const double *src_expansions, int32_t tgt_base_ibox, double *tgt_expansions, void *stream)
{
    if (order < 0 || order > SUMPY_MAX_ORDER) {
        set_last_error("m2l: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    return m2l_f64_launch(ncoeff_of(order), nitems, item_tile, item_group_begin, item_group_end,
                          tile_width, tile_targets, tile_scale, group_class, group_sources,
                          nclasses, class_matrices, src_base_ibox, src_expansions, tgt_base_ibox,
                          tgt_expansions, stream);
}

int sumpy_helmholtz_m2l_translation_classes_f64(
    int order, int32_t nitems, const int32_t *item_tile, const int32_t *item_group_begin,
    const int32_t *item_group_end, int32_t tile_width, const int32_t *tile_targets,
    const double *tile_scale, const int32_t *group_class, const int32_t *group_sources,
    int32_t nclasses, const double *class_matrices, int32_t src_base_ibox,
    const double *src_expansions, int32_t tgt_base_ibox, double *tgt_expansions, void *stream)
{
    if (order < 0 || order > SUMPY_MAX_ORDER) {
        set_last_error("helmholtz m2l: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    return m2l_f64_launch(2 * ncoeff_of(order), nitems, item_tile, item_group_begin,
                          item_group_end, tile_width, tile_targets, tile_scale, group_class,
                          group_sources, nclasses, class_matrices, src_base_ibox, src_expansions,
                          tgt_base_ibox, tgt_expansions, stream);
}

int sumpy_class_gemm_f64(
    int32_t n, int32_t k_split, int32_t nitems, const int32_t *item_tile,
    const int32_t *item_group_begin, const int32_t *item_group_end, int32_t tile_width,
    const int32_t *tile_targets, const double *tile_scale, const int32_t *group_class,
    const int32_t *group_sources, int32_t nclasses, const double *class_matrices,
    int32_t src_base_ibox, const double *src_expansions, int32_t tgt_base_ibox,
    double *tgt_expansions, void *stream)
{
    if (n < 1 || n > 2 * ncoeff_of(SUMPY_MAX_ORDER)) return bad_arg("class gemm: bad n");
    return m2l_f64_launch(n, nitems, item_tile, item_group_begin, item_group_end, tile_width,
                          tile_targets, tile_scale, group_class, group_sources, nclasses,
                          class_matrices, src_base_ibox, src_expansions, tgt_base_ibox,
                          tgt_expansions, stream, k_split);
}

int sumpy_class_gemm_chain_f64(
    int32_t n, int32_t nsteps, const int32_t *step_unit_start, const int32_t *step_item_start,
    const int32_t *step_ksplit, int32_t total_units, const int32_t *item_tile,
    const int32_t *item_group_begin, const int32_t *item_group_end, int32_t tile_width,
    const int32_t *tile_targets, const double *tile_scale, const int32_t *group_class,
    const int32_t *group_sources, const double *class_matrices, double *expansions,
    int32_t *queue, int32_t *status, void *stream)
{
    if (n < 1 || n > 2 * ncoeff_of(SUMPY_MAX_ORDER)) return bad_arg("class gemm chain: bad n");
    if (tile_width != TW) return bad_arg("class gemm chain: tile_width must be 64");
    if (nsteps < 0 || nsteps > CHAIN_MAX_STEPS) return bad_arg("class gemm chain: nsteps in [0, 64]");
    if (total_units < 0) return bad_arg("class gemm chain: negative unit count");
    if (nsteps == 0 || total_units == 0) return SUMPY_OK;
    if (!step_unit_start || !step_item_start || !step_ksplit || !item_tile || !item_group_begin ||
        !item_group_end || !tile_targets || !tile_scale || !group_class || !group_sources ||
        !class_matrices || !expansions || !queue)
        return bad_arg("class gemm chain: null pointer argument");
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int32_t) * (1 + nsteps), st);
    if (e != cudaSuccess) return check_launch("class gemm chain: clearing the queue");
    ChainArgs a;
    a.n = n; a.nsteps = nsteps;
    a.step_unit_start = step_unit_start; a.step_item_start = step_item_start;
    a.step_ksplit = step_ksplit;
    a.item_tile = item_tile; a.item_g0 = item_group_begin; a.item_g1 = item_group_end;
    a.tile_targets = tile_targets; a.tile_scale = tile_scale;
    a.group_class = group_class; a.group_sources = group_sources; a.mats = class_matrices;
    a.expansions = expansions; a.queue = queue; a.status = status;
    a.wait_cycles = wait_cycles_budget();
    int dev = 0, sms = 148, per_sm = 1;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return bad_arg("class gemm chain: no device");
    if (n <= 64) {
        a.nrowblk = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, class_gemm_chain_kernel<64>, 64, 0);
        const int grid = std::max(1, std::min(total_units, sms * std::max(per_sm, 1)));
        class_gemm_chain_kernel<64><<<grid, 64, 0, st>>>(a);
    } else {
        a.nrowblk = (n + 127) / 128;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, class_gemm_chain_kernel<128>, 128, 0);
        const int grid = std::max(1, std::min(total_units, sms * std::max(per_sm, 1)));
        class_gemm_chain_kernel<128><<<grid, 128, 0, st>>>(a);
    }
    return check_launch("class_gemm_chain_kernel");
}

}  // extern "C"
