// M2L per translation class as dense GEMMs (FP64).
//
// sumpy applies M2L per target box and List-2 source with the translation
// class's derivative vector, via FFT or a Toeplitz product
// (sumpy/e2e.py:310-558, sumpy/expansion/m2l.py:363-389, 913-1001). In exact
// arithmetic each class c is the linear map
//     L[t] += (r_tgt/r_src)^|t| sum_s M[s] D_c[s+t]
// so with T_c[t][s] (one n x n matrix per class, built on the host) the
// level's M2L is sum_c T_c * M[:, sources of class c].
//
// Work unit: a tile of 64 target boxes. The host groups the tile's List-2
// entries by class; each group is one GEMM step C += T_c * B_g with B_g the
// gathered source multipoles (one per target slot, zero where absent).
// The accumulator C (rows of the tile x 64 targets) stays in registers over
// all of the tile's groups and is added to the local expansions once.
// A CTA covers ROWS (64 or 128) output rows; more rows use gridDim.y.
// Thread (ty, tx) owns rows ty + (ROWS/8) r and target slots tx + 8 c
// (r, c < 8), so each shared-memory read of a k-step is conflict-free.
#include "common.cuh"

namespace sumpy {
namespace {

constexpr int TW = 64;  // target boxes per tile
constexpr int KC = 16;  // k-chunk

template <int ROWS>
__global__ void __launch_bounds__(ROWS)
m2l_f64_kernel(int n, const int32_t *__restrict__ tile_targets,
               const int32_t *__restrict__ tile_group_starts, const int32_t *__restrict__ group_class,
               const int32_t *__restrict__ group_sources, const double *__restrict__ mats,
               double scale, int32_t sbase, const double *__restrict__ src, int32_t tbase,
               double *__restrict__ tgt)
{
    constexpr int NT = ROWS;          // (ROWS / 8) x 8 threads
    constexpr int RG = ROWS / 8;      // row groups
    __shared__ double As[KC][ROWS + 1];
    __shared__ double Bs[KC][TW + 1];
    __shared__ int32_t srcs[TW];

    const int tile = blockIdx.x;
    const int row0 = blockIdx.y * ROWS;
    const int tid = threadIdx.x;
    const int tx = tid % 8, ty = tid / 8;

    double acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;

    const int g0 = tile_group_starts[tile], g1 = tile_group_starts[tile + 1];
    for (int g = g0; g < g1; ++g) {
        const int cls = group_class[g];
        const double *A = mats + (int64_t)cls * n * n;
        __syncthreads();
        for (int s = tid; s < TW; s += NT) srcs[s] = group_sources[(int64_t)g * TW + s];
        __syncthreads();
        for (int k0 = 0; k0 < n; k0 += KC) {
            for (int idx = tid; idx < ROWS * KC; idx += NT) {
                const int r = idx / KC, kk = idx % KC;
                const int row = row0 + r, k = k0 + kk;
                As[kk][r] = (row < n && k < n) ? A[(int64_t)row * n + k] : 0.0;
            }
            for (int idx = tid; idx < TW * KC; idx += NT) {
                const int slot = idx / KC, kk = idx % KC;
                const int32_t s = srcs[slot];
                const int k = k0 + kk;
                Bs[kk][slot] = (s >= 0 && k < n) ? src[(int64_t)(s - sbase) * n + k] : 0.0;
            }
            __syncthreads();
#pragma unroll 4
            for (int kk = 0; kk < KC; ++kk) {
                double a[8], b[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) a[r] = As[kk][ty + RG * r];
#pragma unroll
                for (int c = 0; c < 8; ++c) b[c] = Bs[kk][tx + 8 * c];
#pragma unroll
                for (int r = 0; r < 8; ++r)
#pragma unroll
                    for (int c = 0; c < 8; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const int32_t t = tile_targets[(int64_t)tile * TW + tx + 8 * c];
        if (t < 0) continue;
        double *o = tgt + (int64_t)(t - tbase) * n;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const int row = row0 + ty + RG * r;
            if (row < n) o[row] += scale * acc[r][c];
        }
    }
}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_m2l_translation_classes_f64(int order, int32_t ntiles, int32_t tile_width,
                                      const int32_t *tile_targets,
                                      const int32_t *tile_group_starts,
                                      const int32_t *group_class, const int32_t *group_sources,
                                      int32_t nclasses, const double *class_matrices,
                                      double matrix_scale, int32_t src_base_ibox,
                                      const double *src_expansions, int32_t tgt_base_ibox,
                                      double *tgt_expansions, void *stream)
{
    if (order < 0 || order > SUMPY_MAX_ORDER) {
        set_last_error("m2l: unsupported order");
        return SUMPY_EUNSUPPORTED;
    }
    if (tile_width != TW) return bad_arg("m2l: tile_width must be 64");
    if (ntiles < 0 || nclasses < 0) return bad_arg("m2l: negative size");
    if (ntiles == 0) return SUMPY_OK;
    if (!tile_targets || !tile_group_starts || !group_class || !group_sources ||
        !class_matrices || !src_expansions || !tgt_expansions)
        return bad_arg("m2l: null pointer argument");
    const int n = ncoeff_of(order);
    cudaStream_t st = as_stream(stream);
    if (n <= 64) {
        dim3 grid(ntiles, 1);
        m2l_f64_kernel<64><<<grid, 64, 0, st>>>(n, tile_targets, tile_group_starts, group_class,
                                                group_sources, class_matrices, matrix_scale,
                                                src_base_ibox, src_expansions, tgt_base_ibox,
                                                tgt_expansions);
    } else {
        dim3 grid(ntiles, (n + 127) / 128);
        m2l_f64_kernel<128><<<grid, 128, 0, st>>>(n, tile_targets, tile_group_starts,
                                                  group_class, group_sources, class_matrices,
                                                  matrix_scale, src_base_ibox, src_expansions,
                                                  tgt_base_ibox, tgt_expansions);
    }
    return check_launch("m2l_f64_kernel");
}

}  // extern "C"
