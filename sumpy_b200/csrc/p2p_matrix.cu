// P2P interaction matrix entries: P2PMatrixGenerator (the dense
// [ntargets, nsources] matrix, sumpy/p2p.py:290-349) and
// P2PMatrixSubsetGenerator (entries at given (target, source) index pairs,
// sumpy/p2p.py:354-477), for the 3D Laplace kernel 1/r and the 3D Helmholtz
// kernel e^{ikr}/r, times the kernel's scaling; with exclude_self the
// entries with source == target_to_source[target] are zero (p2p.py:162-170,
// 322-323, 397-398). FP64; Helmholtz entries are interleaved (re, im) pairs.
//
// Both kernels only write (8 or 16 bytes per entry): the dense matrix is
// HBM-write bound. A CTA covers 8 rows x 128 columns; the 128 sources'
// coordinates are staged in shared memory once and each warp writes 32
// consecutive entries of a row per instruction.
#include <algorithm>

#include "common.cuh"

namespace sumpy {
namespace {

constexpr int MAT_COLS = 128;   // sources per CTA
constexpr int MAT_ROWS = 8;     // rows per CTA pass (one per warp)

template <bool HELM>
__device__ __forceinline__ void pair_entry(double dx, double dy, double dz, double k, double scale,
                                           double &re, double &im)
{
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double ri = rsqrt(r2);
    if (HELM) {
        double sn, cs;
        sincos(k * (r2 * ri), &sn, &cs);
        re = scale * cs * ri;
        im = scale * sn * ri;
    } else {
        re = scale * ri;
        im = 0.0;
    }
}

template <bool HELM>
__global__ void __launch_bounds__(32 * MAT_ROWS)
p2p_matrix_kernel(int64_t ntgt, const double *__restrict__ targets, int64_t tstride,
                  int64_t nsrc, const double *__restrict__ sources, int64_t sstride,
                  const int32_t *__restrict__ target_to_source, double k, double scale,
                  double *__restrict__ result)
{
    __shared__ double sxyz[3][MAT_COLS];
    const int64_t c0 = (int64_t)blockIdx.x * MAT_COLS;
    const int lane = threadIdx.x, row = threadIdx.y;
    const int tid = row * 32 + lane;
    if (tid < MAT_COLS && c0 + tid < nsrc) {
        sxyz[0][tid] = sources[c0 + tid];
        sxyz[1][tid] = sources[sstride + c0 + tid];
        sxyz[2][tid] = sources[2 * sstride + c0 + tid];
    }
    __syncthreads();
    for (int64_t t = (int64_t)blockIdx.y * MAT_ROWS + row; t < ntgt;
         t += (int64_t)gridDim.y * MAT_ROWS) {
        const double tx = targets[t], ty = targets[tstride + t], tz = targets[2 * tstride + t];
        const int64_t self = target_to_source ? (int64_t)target_to_source[t] : -1;
#pragma unroll
        for (int j = 0; j < MAT_COLS / 32; ++j) {
            const int cl = lane + 32 * j;
            const int64_t c = c0 + cl;
            if (c >= nsrc) break;
            double re = 0.0, im = 0.0;
            if (c != self)
                pair_entry<HELM>(tx - sxyz[0][cl], ty - sxyz[1][cl], tz - sxyz[2][cl], k, scale,
                                 re, im);
            const int64_t e = t * nsrc + c;
            if (HELM)
                reinterpret_cast<double2 *>(result)[e] = make_double2(re, im);
            else
                result[e] = re;
        }
    }
}

template <bool HELM>
__global__ void __launch_bounds__(256)
p2p_subset_kernel(int64_t nresult, const int32_t *__restrict__ tgtindices,
                  const int32_t *__restrict__ srcindices, const double *__restrict__ targets,
                  int64_t tstride, const double *__restrict__ sources, int64_t sstride,
                  const int32_t *__restrict__ target_to_source, double k, double scale,
                  double *__restrict__ result)
{
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nresult;
         m += (int64_t)gridDim.x * blockDim.x) {
        const int32_t it = tgtindices[m], is = srcindices[m];
        double re = 0.0, im = 0.0;
        if (!(target_to_source && target_to_source[it] == is))
            pair_entry<HELM>(targets[it] - sources[is], targets[tstride + it] - sources[sstride + is],
                             targets[2 * tstride + it] - sources[2 * sstride + is], k, scale,
                             re, im);
        if (HELM)
            reinterpret_cast<double2 *>(result)[m] = make_double2(re, im);
        else
            result[m] = re;
    }
}

template <bool HELM>
int launch_matrix(int64_t ntargets, const double *targets, int64_t target_stride,
                  int64_t nsources, const double *sources, int64_t source_stride,
                  const int32_t *target_to_source, double k, double scale, double *result,
                  void *stream)
{
    if (ntargets < 0 || nsources < 0) return bad_arg("p2p matrix: negative size");
    if (ntargets == 0 || nsources == 0) return SUMPY_OK;
    if (!targets || !sources || !result) return bad_arg("p2p matrix: null pointer argument");
    if (HELM && (reinterpret_cast<uintptr_t>(result) & 15))
        return bad_arg("p2p matrix: complex result must be 16-byte aligned");
    const int64_t bx = (nsources + MAT_COLS - 1) / MAT_COLS;
    if (bx > INT32_MAX) return bad_arg("p2p matrix: too many sources");
    const int64_t by = std::min<int64_t>((ntargets + MAT_ROWS - 1) / MAT_ROWS, 65535);
    dim3 grid((unsigned)bx, (unsigned)by), block(32, MAT_ROWS);
    p2p_matrix_kernel<HELM><<<grid, block, 0, as_stream(stream)>>>(
        ntargets, targets, target_stride, nsources, sources, source_stride, target_to_source, k,
        scale, result);
    return check_launch("p2p_matrix_kernel");
}

template <bool HELM>
int launch_subset(int64_t nresult, const int32_t *tgtindices, const int32_t *srcindices,
                  const double *targets, int64_t target_stride, const double *sources,
                  int64_t source_stride, const int32_t *target_to_source, double k, double scale,
                  double *result, void *stream)
{
    if (nresult < 0) return bad_arg("p2p matrix subset: negative size");
    if (nresult == 0) return SUMPY_OK;
    if (!tgtindices || !srcindices || !targets || !sources || !result)
        return bad_arg("p2p matrix subset: null pointer argument");
    if (HELM && (reinterpret_cast<uintptr_t>(result) & 15))
        return bad_arg("p2p matrix subset: complex result must be 16-byte aligned");
    const int64_t blocks = std::min<int64_t>((nresult + 255) / 256, 148 * 32);
    p2p_subset_kernel<HELM><<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(
        nresult, tgtindices, srcindices, targets, target_stride, sources, source_stride,
        target_to_source, k, scale, result);
    return check_launch("p2p_subset_kernel");
}

}  // namespace
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_p2p_matrix_f64(int64_t ntargets, const double *targets, int64_t target_stride,
                         int64_t nsources, const double *sources, int64_t source_stride,
                         const int32_t *target_to_source, double scale, double *result,
                         void *stream)
{
    return launch_matrix<false>(ntargets, targets, target_stride, nsources, sources,
                                source_stride, target_to_source, 0.0, scale, result, stream);
}

int sumpy_helmholtz_p2p_matrix_f64(int64_t ntargets, const double *targets,
                                   int64_t target_stride, int64_t nsources,
                                   const double *sources, int64_t source_stride,
                                   const int32_t *target_to_source, double k, double scale,
                                   double *result, void *stream)
{
    return launch_matrix<true>(ntargets, targets, target_stride, nsources, sources,
                               source_stride, target_to_source, k, scale, result, stream);
}

int sumpy_p2p_matrix_subset_f64(int64_t nresult, const int32_t *tgtindices,
                                const int32_t *srcindices, const double *targets,
                                int64_t target_stride, const double *sources,
                                int64_t source_stride, const int32_t *target_to_source,
                                double scale, double *result, void *stream)
{
    return launch_subset<false>(nresult, tgtindices, srcindices, targets, target_stride, sources,
                                source_stride, target_to_source, 0.0, scale, result, stream);
}

int sumpy_helmholtz_p2p_matrix_subset_f64(int64_t nresult, const int32_t *tgtindices,
                                          const int32_t *srcindices, const double *targets,
                                          int64_t target_stride, const double *sources,
                                          int64_t source_stride,
                                          const int32_t *target_to_source, double k,
                                          double scale, double *result, void *stream)
{
    return launch_subset<true>(nresult, tgtindices, srcindices, targets, target_stride, sources,
                               source_stride, target_to_source, k, scale, result, stream);
}

}  // extern "C"
