// Octree, FMM interaction lists and translation classes built on the GPU.
//
// boxtree's role for sumpy (TreeBuilder, FMMTraversalBuilder and
// TranslationClassesBuilder, called at sumpy/fmm.py:356-363; the arrays the
// wrangler consumes are listed at sumpy/fmm.py:372-397, 543-592, 609-1083).
// The definitions are those of the host builder (sumpy_b200/csrc/tree.cpp),
// and the results are the same arrays, bit for bit: a box is refined while it
// holds more than max_particles_in_box particles, empty children are not
// created, boxes are numbered level by level in Morton order, particles are
// sorted by Morton key (stable), and Lists 1-4 and the translation classes
// follow the adaptive FMM with one-box separation.
//
// A build can hold several independent problems (a forest): problem p owns
// the particle range [starts[p], starts[p+1]) of the user arrays, every
// problem gets its own root box at level 0 in the common root geometry, and
// boxes are numbered level by level, problem after problem, Morton order
// inside a problem -- the layout of sumpy_b200.forest.merge_trees. Lists
// never cross problems. One problem is the ordinary tree.
//
// Phases (all on the caller's stream; the host waits only for the few
// scalars that size the next phase):
//   1. bounding box (min/max reduction; skipped when the caller fixes it)
//   2. Morton keys and a stable sort of each problem's particles (CUB radix
//      sort, segmented by problem)
//   3. levels: per level, octant bounds of every box by binary search in the
//      sorted keys, child counts, a scan, the children -- one D2H count per
//      level
//   4. box attributes, box sets (stream compaction), colleagues per level
//   5. Lists 1/3 (leaf target boxes) and 2/4 (target-or-target-parent boxes):
//      a counting pass, a scan, a filling pass that sorts each list
//   6. List 3 regrouped by source level
// Every index is checked against its array's extent before use; a list
// traversal that would overflow its fixed-size stack reports an error.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"

namespace sumpy {
namespace gtree {

constexpr int KEY_BITS = 21;
constexpr int NCLASSES = 316;
constexpr int MAXCOLL = 27;
constexpr int STACK = 512;

// {{{ device buffers

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaStream_t st = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes), st(o.st) { o.p = nullptr; o.bytes = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept
    {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; st = o.st; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

struct Fail {
    std::string msg;
};

inline void ck(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw Fail{std::string(what) + ": " + cudaGetErrorString(e)};
}

inline DevBuf dalloc(size_t bytes, cudaStream_t st)
{
    DevBuf b;
    b.st = st;
    b.bytes = bytes;
    if (bytes) ck(cudaMallocAsync(&b.p, bytes, st), "cudaMallocAsync");
    return b;
}

template <class T> inline DevBuf dalloc_n(int64_t n, cudaStream_t st)
{
    return dalloc(sizeof(T) * (size_t)std::max<int64_t>(n, 0), st);
}

inline unsigned nblocks(int64_t n, int threads = 256)
{
    const int64_t b = (n + threads - 1) / threads;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 1 << 30));
}

inline void launched(const char *what) { ck(cudaGetLastError(), what); }

// }}}

// {{{ bounding box and keys

// per-dimension min / max of the finite coordinates and a count of the
// non-finite ones: each block reduces its share into partial[block][7]
// (min x3, max x3, count as a double), one block combines the partials
__global__ void bbox_partial_kernel(int64_t n, const double *__restrict__ x,
                                    const double *__restrict__ y, const double *__restrict__ z,
                                    double *__restrict__ partial)
{
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    double bad = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double p[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (!isfinite(p[d])) { bad += 1; continue; }
            lo[d] = fmin(lo[d], p[d]);
            hi[d] = fmax(hi[d], p[d]);
        }
    }
    typedef cub::BlockReduce<double, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    double r[7];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        r[d] = BR(tmp).Reduce(lo[d], cub::Min());
        __syncthreads();
        r[3 + d] = BR(tmp).Reduce(hi[d], cub::Max());
        __syncthreads();
    }
    r[6] = BR(tmp).Sum(bad);
    if (threadIdx.x == 0)
        for (int k = 0; k < 7; ++k) partial[7 * (int64_t)blockIdx.x + k] = r[k];
}

// combine nparts partials (one block of 256 threads) into out[0..6]
__global__ void bbox_combine_kernel(int nparts, const double *__restrict__ partial,
                                    double *__restrict__ out)
{
    double r[7] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY, 0};
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        const double *q = partial + 7 * (int64_t)i;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            r[d] = fmin(r[d], q[d]);
            r[3 + d] = fmax(r[3 + d], q[3 + d]);
        }
        r[6] += q[6];
    }
    typedef cub::BlockReduce<double, 256> BR;
    __shared__ typename BR::TempStorage tmp;
    double o[7];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        o[d] = BR(tmp).Reduce(r[d], cub::Min());
        __syncthreads();
        o[3 + d] = BR(tmp).Reduce(r[3 + d], cub::Max());
        __syncthreads();
    }
    o[6] = BR(tmp).Sum(r[6]);
    if (threadIdx.x == 0)
        for (int k = 0; k < 7; ++k) out[k] = o[k];
}

__device__ __forceinline__ uint64_t spread3(uint32_t v)
{
    uint64_t x = v & 0x1fffff;
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

// Morton key of each particle; also counts particles outside a caller-fixed
// root box. (p - bmin) * scale is a subtraction then a product (nothing to
// contract), floor and the clamp are exact: the keys equal the host's.
__global__ void keys_kernel(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                            const double *__restrict__ z, double b0, double b1, double b2,
                            double scale, double extent, int check_box, uint64_t *__restrict__ keys,
                            int32_t *__restrict__ idx, unsigned long long *outside)
{
    const uint32_t maxc = (1u << KEY_BITS) - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double p[3] = {x[i], y[i], z[i]};
        const double bm[3] = {b0, b1, b2};
        uint32_t q[3];
        bool out = false;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (check_box && (p[d] < bm[d] || p[d] > __dadd_rn(bm[d], extent))) out = true;
            double v = floor(__dmul_rn(__dsub_rn(p[d], bm[d]), scale));
            if (v < 0) v = 0;
            if (v > (double)maxc) v = (double)maxc;
            q[d] = (uint32_t)v;
        }
        if (out) atomicAdd(outside, 1ull);
        keys[i] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
        idx[i] = (int32_t)i;
    }
}

// stable sort of (key, index) pairs inside each problem's segment
void sort_segments(int64_t n, DevBuf &keys, DevBuf &idx, const std::vector<int64_t> &starts,
                   cudaStream_t st, DevBuf &keys_out, DevBuf &idx_out)
{
    keys_out = dalloc_n<uint64_t>(n, st);
    idx_out = dalloc_n<int32_t>(n, st);
    if (n == 0) return;
    const int nseg = (int)starts.size() - 1;
    size_t tmp_bytes = 0;
    if (nseg == 1) {
        ck(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys.as<uint64_t>(),
                                           keys_out.as<uint64_t>(), idx.as<int32_t>(),
                                           idx_out.as<int32_t>(), (int)n, 0, 3 * KEY_BITS, st),
           "cub sort (size)");
        DevBuf tmp = dalloc(tmp_bytes, st);
        ck(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, keys.as<uint64_t>(),
                                           keys_out.as<uint64_t>(), idx.as<int32_t>(),
                                           idx_out.as<int32_t>(), (int)n, 0, 3 * KEY_BITS, st),
           "cub sort");
        return;
    }
    std::vector<int32_t> off(starts.begin(), starts.end());
    DevBuf doff = dalloc_n<int32_t>(nseg + 1, st);
    ck(cudaMemcpyAsync(doff.p, off.data(), sizeof(int32_t) * off.size(), cudaMemcpyHostToDevice, st),
       "copy segment offsets");
    const int32_t *b = doff.as<int32_t>();
    ck(cub::DeviceSegmentedRadixSort::SortPairs(nullptr, tmp_bytes, keys.as<uint64_t>(),
                                                keys_out.as<uint64_t>(), idx.as<int32_t>(),
                                                idx_out.as<int32_t>(), (int)n, nseg, b, b + 1, 0,
                                                3 * KEY_BITS, st),
       "cub segmented sort (size)");
    DevBuf tmp = dalloc(tmp_bytes, st);
    ck(cub::DeviceSegmentedRadixSort::SortPairs(tmp.p, tmp_bytes, keys.as<uint64_t>(),
                                                keys_out.as<uint64_t>(), idx.as<int32_t>(),
                                                idx_out.as<int32_t>(), (int)n, nseg, b, b + 1, 0,
                                                3 * KEY_BITS, st),
       "cub segmented sort");
    // (the offsets and the scratch are released in stream order, after the sort)
}

// }}}

// {{{ scans

__global__ void write_starts_kernel(int64_t n, const int64_t *__restrict__ incl,
                                    int32_t *__restrict__ starts, int64_t *__restrict__ total)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
         i += (int64_t)gridDim.x * blockDim.x) {
        starts[i] = i == 0 ? 0 : (int32_t)incl[i - 1];
        if (i == n && total) *total = n == 0 ? 0 : incl[n - 1];
    }
}

struct ToI64 {
    __host__ __device__ int64_t operator()(int32_t v) const { return (int64_t)v; }
};

// starts[0] = 0, starts[i + 1] = cnt[0] + ... + cnt[i] (int32, n + 1
// entries); the total goes to *dtotal (device) without waiting for it
void scan_counts_async(const int32_t *cnt, int64_t n, DevBuf &starts, int64_t *dtotal,
                       cudaStream_t st)
{
    starts = dalloc_n<int32_t>(n + 1, st);
    DevBuf incl = dalloc_n<int64_t>(std::max<int64_t>(n, 1), st);
    if (n > 0) {
        thrust::transform_iterator<ToI64, const int32_t *, int64_t> it(cnt, ToI64());
        size_t tmp_bytes = 0;
        ck(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, it, incl.as<int64_t>(), (int)n, st),
           "cub scan (size)");
        DevBuf tmp = dalloc(tmp_bytes, st);
        ck(cub::DeviceScan::InclusiveSum(tmp.p, tmp_bytes, it, incl.as<int64_t>(), (int)n, st),
           "cub scan");
    }
    write_starts_kernel<<<nblocks(n + 1), 256, 0, st>>>(n, incl.as<int64_t>(), starts.as<int32_t>(),
                                                        dtotal);
    launched("write_starts_kernel");
}

// host copies of n device int64 values (one wait); each must fit int32
std::vector<int64_t> read_totals(const DevBuf &dtot, int n, cudaStream_t st)
{
    std::vector<int64_t> h(n);
    ck(cudaMemcpyAsync(h.data(), dtot.p, 8 * (size_t)n, cudaMemcpyDeviceToHost, st), "copy totals");
    ck(cudaStreamSynchronize(st), "scan");
    for (int64_t v : h)
        if (v > INT32_MAX) throw Fail{"list or box count exceeds int32"};
    return h;
}

int64_t scan_counts(const int32_t *cnt, int64_t n, DevBuf &starts, cudaStream_t st)
{
    DevBuf dtot = dalloc_n<int64_t>(1, st);
    scan_counts_async(cnt, n, starts, dtot.as<int64_t>(), st);
    return read_totals(dtot, 1, st)[0];
}

// }}}

// {{{ levels

struct Level {
    int64_t n = 0;
    DevBuf c[3], slo, shi, tlo, thi, parent, child;   // child: [n][8], -1 none
};

__device__ __forceinline__ int octant_of(uint64_t key, int child_level)
{
    return (int)((key >> (3 * (KEY_BITS - child_level))) & 7);
}

// first index in [lo, hi) whose octant at child_level is >= oct
__device__ int32_t octant_bound(const uint64_t *__restrict__ keys, int32_t lo, int32_t hi,
                                int child_level, int oct)
{
    while (lo < hi) {
        const int32_t mid = lo + (hi - lo) / 2;
        if (octant_of(keys[mid], child_level) < oct) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

struct LevelPtrs {
    const int32_t *c0, *c1, *c2, *slo, *shi, *tlo, *thi;
};

__global__ void split_count_kernel(int64_t n, LevelPtrs b, int level, int allow, int sat,
                                   int max_particles, const uint64_t *__restrict__ skeys,
                                   const uint64_t *__restrict__ tkeys, int32_t *__restrict__ nchild,
                                   int32_t *__restrict__ bounds)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t slo = b.slo[i], shi = b.shi[i], tlo = b.tlo[i], thi = b.thi[i];
        const int64_t count = (int64_t)(shi - slo) + (sat ? 0 : (int64_t)(thi - tlo));
        int32_t *bd = bounds + 18 * i;
        if (!allow || count <= max_particles) {
            nchild[i] = 0;
            continue;
        }
        bd[0] = slo; bd[8] = shi; bd[9] = tlo; bd[17] = thi;
        for (int o = 1; o < 8; ++o) {
            bd[o] = octant_bound(skeys, slo, shi, level + 1, o);
            bd[9 + o] = octant_bound(tkeys, tlo, thi, level + 1, o);
        }
        int nc = 0;
        for (int o = 0; o < 8; ++o)
            if (bd[o + 1] != bd[o] || bd[10 + o] != bd[9 + o]) ++nc;
        nchild[i] = nc;
    }
}

struct LevelOut {
    int32_t *c0, *c1, *c2, *slo, *shi, *tlo, *thi, *parent;
};

__global__ void split_fill_kernel(int64_t n, LevelPtrs b, const int32_t *__restrict__ nchild,
                                  const int32_t *__restrict__ bounds,
                                  const int32_t *__restrict__ off, int64_t n_next,
                                  int32_t base_this, int32_t base_next, LevelOut o,
                                  int32_t *__restrict__ child)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        int32_t *ch = child + 8 * i;
        for (int q = 0; q < 8; ++q) ch[q] = -1;
        if (nchild[i] == 0) continue;
        const int32_t *bd = bounds + 18 * i;
        int32_t j = off[i];
        for (int q = 0; q < 8; ++q) {
            if (bd[q + 1] == bd[q] && bd[10 + q] == bd[9 + q]) continue;
            if (j < 0 || j >= n_next) continue;   // cannot happen: the scan sized the level
            o.c0[j] = 2 * b.c0[i] + ((q >> 2) & 1);
            o.c1[j] = 2 * b.c1[i] + ((q >> 1) & 1);
            o.c2[j] = 2 * b.c2[i] + (q & 1);
            o.slo[j] = bd[q]; o.shi[j] = bd[q + 1];
            o.tlo[j] = bd[9 + q]; o.thi[j] = bd[10 + q];
            o.parent[j] = base_this + (int32_t)i;
            ch[q] = base_next + j;
            ++j;
        }
    }
}

inline LevelPtrs ptrs(const Level &L)
{
    return {L.c[0].as<int32_t>(), L.c[1].as<int32_t>(), L.c[2].as<int32_t>(), L.slo.as<int32_t>(),
            L.shi.as<int32_t>(), L.tlo.as<int32_t>(), L.thi.as<int32_t>()};
}

void alloc_level(Level &L, int64_t n, cudaStream_t st)
{
    L.n = n;
    for (int d = 0; d < 3; ++d) L.c[d] = dalloc_n<int32_t>(n, st);
    L.slo = dalloc_n<int32_t>(n, st); L.shi = dalloc_n<int32_t>(n, st);
    L.tlo = dalloc_n<int32_t>(n, st); L.thi = dalloc_n<int32_t>(n, st);
    L.parent = dalloc_n<int32_t>(n, st);
}

// }}}

// {{{ boxes

struct BoxPtrs {
    const int32_t *level, *c0, *c1, *c2, *slo, *shi, *tlo, *thi, *parent, *child;  // child [nb][8]
    const uint8_t *leaf;
    int64_t nb;
};

// One 64-byte record per box for the list traversals: a visit touches one
// cache line instead of one line per attribute array.
struct __align__(64) Rec {
    int32_t c0, c1, c2, level, nsrc, flags, parent, pad;   // flags: 1 = leaf
    int32_t child[8];                                      // -1: none
};
static_assert(sizeof(Rec) == 64, "box record size");

__device__ __forceinline__ Rec load_rec(const Rec *__restrict__ R, int32_t b)
{
    const int4 *p = reinterpret_cast<const int4 *>(R + b);
    Rec r;
    int4 *q = reinterpret_cast<int4 *>(&r);
#pragma unroll
    for (int k = 0; k < 4; ++k) q[k] = __ldg(p + k);
    return r;
}

__device__ __forceinline__ bool rec_adjacent(const Rec &a, const Rec &b)
{
    const int sa = KEY_BITS - a.level, sb = KEY_BITS - b.level;
    const int32_t ca[3] = {a.c0, a.c1, a.c2}, cb[3] = {b.c0, b.c1, b.c2};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int64_t la = (int64_t)ca[d] << sa, lb = (int64_t)cb[d] << sb;
        if (la > lb + ((int64_t)1 << sb) || lb > la + ((int64_t)1 << sa)) return false;
    }
    return true;
}

__global__ void pack_records_kernel(BoxPtrs B, Rec *__restrict__ R)
{
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B.nb;
         b += (int64_t)gridDim.x * blockDim.x) {
        Rec r;
        r.c0 = B.c0[b]; r.c1 = B.c1[b]; r.c2 = B.c2[b]; r.level = B.level[b];
        r.nsrc = B.shi[b] - B.slo[b];
        r.flags = B.leaf[b] ? 1 : 0;
        r.parent = B.parent[b];
        r.pad = 0;
        for (int o = 0; o < 8; ++o) r.child[o] = B.child[8 * b + o];
        R[b] = r;
    }
}

__global__ void leaf_kernel(int64_t nb, const int32_t *__restrict__ child, uint8_t *__restrict__ leaf)
{
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
         b += (int64_t)gridDim.x * blockDim.x) {
        bool l = true;
        for (int o = 0; o < 8; ++o) l = l && child[8 * b + o] < 0;
        leaf[b] = l ? 1 : 0;
    }
}

// centers (bbox_min + (c + 1/2) h, a rounded product then a rounded sum, as
// on the host), boxtree-shaped attribute arrays and the box-set flags
__global__ void attrs_kernel(BoxPtrs B, double b0, double b1, double b2, double root_extent,
                             double *__restrict__ centers,
                             int32_t *__restrict__ levels, int32_t *__restrict__ parent_out,
                             int32_t *__restrict__ child_out, int32_t *__restrict__ coords,
                             int32_t *__restrict__ sstart, int32_t *__restrict__ scum,
                             int32_t *__restrict__ snc, int32_t *__restrict__ tstart,
                             int32_t *__restrict__ tcum, int32_t *__restrict__ tnc,
                             uint8_t *__restrict__ f_src, uint8_t *__restrict__ f_tgt,
                             uint8_t *__restrict__ f_sparent, uint8_t *__restrict__ f_ttp)
{
    const int64_t nb = B.nb;
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb;
         b += (int64_t)gridDim.x * blockDim.x) {
        const int lev = B.level[b];
        const double h = root_extent / (double)(1LL << lev);
        const int32_t c[3] = {B.c0[b], B.c1[b], B.c2[b]};
        const double bm[3] = {b0, b1, b2};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            centers[d * nb + b] = __dadd_rn(bm[d], __dmul_rn((double)c[d] + 0.5, h));
            coords[d * nb + b] = c[d];
        }
        levels[b] = lev;
        parent_out[b] = lev == 0 ? (int32_t)b : B.parent[b];   // a root is its own parent
        const bool leaf = B.leaf[b] != 0;
        for (int o = 0; o < 8; ++o) {
            const int32_t ch = B.child[8 * b + o];
            child_out[(int64_t)o * nb + b] = ch < 0 ? 0 : ch;
        }
        const int32_t ns = B.shi[b] - B.slo[b], nt = B.thi[b] - B.tlo[b];
        sstart[b] = B.slo[b]; scum[b] = ns; snc[b] = leaf ? ns : 0;
        tstart[b] = B.tlo[b]; tcum[b] = nt; tnc[b] = leaf ? nt : 0;
        f_src[b] = leaf && ns > 0;
        f_tgt[b] = leaf && nt > 0;
        f_sparent[b] = !leaf && ns > 0;
        f_ttp[b] = nt > 0;
    }
}

// colleagues of the boxes [b0, b1) of one level: the same-level boxes that
// touch them (self included), from the parent's colleagues' children, in
// increasing box number (by induction from the root's list {root})
__global__ void colleagues_kernel(const Rec *__restrict__ R, int32_t b0, int32_t b1,
                                  int32_t *__restrict__ coll, int32_t *__restrict__ ncoll,
                                  int32_t *__restrict__ err)
{
    for (int64_t b = b0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < b1;
         b += (int64_t)gridDim.x * blockDim.x) {
        const Rec rb = load_rec(R, (int32_t)b);
        int n = 0;
        if (rb.level == 0) {
            coll[MAXCOLL * b] = (int32_t)b;
            n = 1;
        } else {
            const int32_t par = rb.parent;
            const int np = ncoll[par];
            for (int k = 0; k < np; ++k) {
                const Rec rp = load_rec(R, coll[MAXCOLL * (int64_t)par + k]);
                for (int o = 0; o < 8; ++o) {
                    const int32_t c = rp.child[o];
                    if (c < 0 || !rec_adjacent(load_rec(R, c), rb)) continue;
                    if (n < MAXCOLL) coll[MAXCOLL * b + n] = c;
                    else atomicExch(err, 1);
                    ++n;
                }
            }
        }
        ncoll[b] = n < MAXCOLL ? n : MAXCOLL;
    }
}

// }}}

// {{{ interaction lists

__constant__ int16_t c_class_of[343];   // rank of (vx, vy, vz) in [-3,3]^3 \ [-1,1]^3, or -1

__device__ __forceinline__ void sort_segment(int32_t *a, int n)
{
    for (int i = 1; i < n; ++i) {
        const int32_t v = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; --j; }
        a[j + 1] = v;
    }
}

// pairs (box, class) sorted by box
__device__ __forceinline__ void sort_segment2(int32_t *a, int32_t *c, int n)
{
    for (int i = 1; i < n; ++i) {
        const int32_t v = a[i], w = c[i];
        int j = i - 1;
        while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; c[j + 1] = c[j]; --j; }
        a[j + 1] = v;
        c[j + 1] = w;
    }
}

// List 1 and List 3 of each leaf target box. fill == 0: count into n1, n3;
// fill == 1: write at the offsets s1, s3 and sort each list.
__global__ void lists13_kernel(const Rec *__restrict__ R, const int32_t *__restrict__ coll,
                               const int32_t *__restrict__ ncoll, int64_t ntb,
                               const int32_t *__restrict__ tboxes, int fill,
                               int32_t *__restrict__ n1, int32_t *__restrict__ n3,
                               const int32_t *__restrict__ s1, const int32_t *__restrict__ s3,
                               int32_t *__restrict__ l1, int32_t *__restrict__ l3,
                               int32_t *__restrict__ err)
{
    for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < ntb;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int32_t t = tboxes[it];
        const Rec rt = load_rec(R, t);
        int32_t stack[STACK];
        int sp = 0;
        int c1 = 0, c3 = 0;
        int32_t *o1 = fill ? l1 + s1[it] : nullptr;
        int32_t *o3 = fill ? l3 + s3[it] : nullptr;
        const int cap1 = fill ? s1[it + 1] - s1[it] : 0;
        const int cap3 = fill ? s3[it + 1] - s3[it] : 0;
        for (int k = 0; k < ncoll[t]; ++k) stack[sp++] = coll[MAXCOLL * (int64_t)t + k];
        bool overflow = false;
        while (sp > 0) {
            const int32_t c = stack[--sp];
            const Rec rc = load_rec(R, c);
            if (rc.flags & 1) {
                if (rc.nsrc > 0) {
                    if (fill && c1 < cap1) o1[c1] = c;
                    ++c1;
                }
                continue;
            }
            for (int o = 0; o < 8; ++o) {
                const int32_t d = rc.child[o];
                if (d < 0) continue;
                const Rec rd = load_rec(R, d);
                if (rec_adjacent(rd, rt)) {
                    if (sp < STACK) stack[sp++] = d;
                    else overflow = true;
                } else if (rd.nsrc > 0) {
                    if (fill && c3 < cap3) o3[c3] = d;
                    ++c3;
                }
            }
        }
        // coarser leaves touching t: leaf colleagues of its ancestors
        if (rt.level > 0) {
            for (int32_t a = rt.parent;;) {
                const Rec ra = load_rec(R, a);
                for (int k = 0; k < ncoll[a]; ++k) {
                    const int32_t c = coll[MAXCOLL * (int64_t)a + k];
                    if (c == a) continue;
                    const Rec rc = load_rec(R, c);
                    if ((rc.flags & 1) && rc.nsrc > 0 && rec_adjacent(rc, rt)) {
                        if (fill && c1 < cap1) o1[c1] = c;
                        ++c1;
                    }
                }
                if (ra.level == 0) break;
                a = ra.parent;
            }
        }
        if (overflow) atomicExch(err, 2);
        if (fill) {
            if (c1 != cap1 || c3 != cap3) atomicExch(err, 3);
            sort_segment(o1, c1 < cap1 ? c1 : cap1);
            sort_segment(o3, c3 < cap3 ? c3 : cap3);
        } else {
            n1[it] = c1;
            n3[it] = c3;
        }
    }
}

// List 2 (with the global translation class of each entry) and List 4 of
// each target-or-target-parent box; same two modes.
__global__ void lists24_kernel(const Rec *__restrict__ R, const int32_t *__restrict__ coll,
                               const int32_t *__restrict__ ncoll, int64_t nttp,
                               const int32_t *__restrict__ ttp, int fill,
                               int32_t *__restrict__ n2, int32_t *__restrict__ n4,
                               const int32_t *__restrict__ s2, const int32_t *__restrict__ s4,
                               int32_t *__restrict__ l2, int32_t *__restrict__ l2cls,
                               int32_t *__restrict__ l4, int32_t *__restrict__ err)
{
    for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < nttp;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = ttp[it];
        const Rec rb = load_rec(R, b);
        const int lev = rb.level;
        int c2 = 0, c4 = 0;
        int32_t *o2 = fill ? l2 + s2[it] : nullptr;
        int32_t *oc = fill ? l2cls + s2[it] : nullptr;
        int32_t *o4 = fill ? l4 + s4[it] : nullptr;
        const int cap2 = fill ? s2[it + 1] - s2[it] : 0;
        const int cap4 = fill ? s4[it + 1] - s4[it] : 0;
        if (lev >= 1) {
            const int32_t par = rb.parent;
            const Rec rpar = load_rec(R, par);
            if (lev >= 2) {
                for (int k = 0; k < ncoll[par]; ++k) {
                    const Rec rpc = load_rec(R, coll[MAXCOLL * (int64_t)par + k]);
                    for (int o = 0; o < 8; ++o) {
                        const int32_t d = rpc.child[o];
                        if (d < 0) continue;
                        const Rec rd = load_rec(R, d);
                        if (rd.nsrc <= 0) continue;
                        const int v0 = rb.c0 - rd.c0, v1 = rb.c1 - rd.c1, v2 = rb.c2 - rd.c2;
                        if (abs(v0) <= 1 && abs(v1) <= 1 && abs(v2) <= 1) continue;
                        int cls = -1;
                        if (abs(v0) <= 3 && abs(v1) <= 3 && abs(v2) <= 3)
                            cls = c_class_of[((v0 + 3) * 7 + (v1 + 3)) * 7 + (v2 + 3)];
                        if (cls < 0) atomicExch(err, 4);
                        if (fill && c2 < cap2) {
                            o2[c2] = d;
                            oc[c2] = (lev - 2) * NCLASSES + cls;
                        }
                        ++c2;
                    }
                }
            }
            for (int32_t a = par;;) {
                const Rec ra = load_rec(R, a);
                for (int k = 0; k < ncoll[a]; ++k) {
                    const int32_t c = coll[MAXCOLL * (int64_t)a + k];
                    if (c == a) continue;
                    const Rec rc = load_rec(R, c);
                    if ((rc.flags & 1) && rc.nsrc > 0 && rec_adjacent(rc, rpar) &&
                        !rec_adjacent(rc, rb)) {
                        if (fill && c4 < cap4) o4[c4] = c;
                        ++c4;
                    }
                }
                if (ra.level == 0) break;
                a = ra.parent;
            }
        }
        if (fill) {
            if (c2 != cap2 || c4 != cap4) atomicExch(err, 3);
            sort_segment2(o2, oc, c2 < cap2 ? c2 : cap2);
            sort_segment(o4, c4 < cap4 ? c4 : cap4);
        } else {
            n2[it] = c2;
            n4[it] = c4;
        }
    }
}

// For every target box and every source level: the first entry and the
// number of entries of its (sorted) List 3 on that level -- box numbers are
// level-major, so one level is one range of the list.
__global__ void l3_levels_kernel(int64_t ntb, int nl, const int32_t *__restrict__ s3,
                                 const int32_t *__restrict__ l3,
                                 const int32_t *__restrict__ level_start,
                                 int32_t *__restrict__ first2d, int32_t *__restrict__ cnt2d,
                                 uint8_t *__restrict__ flag2d)
{
    for (int64_t it = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; it < ntb;
         it += (int64_t)gridDim.x * blockDim.x) {
        const int32_t a = s3[it], e = s3[it + 1];
        int l = 0;
        int32_t j = a;
        for (; l < nl; ++l) {
            const int32_t f = j;
            while (j < e && l3[j] < level_start[l + 1]) ++j;
            first2d[(int64_t)l * ntb + it] = f;
            cnt2d[(int64_t)l * ntb + it] = j - f;
            flag2d[(int64_t)l * ntb + it] = j > f;
        }
    }
}

// per selected (level, target) k: its count, target box and first entry
__global__ void l3_selected_kernel(int64_t nsel, int64_t ntb, const int32_t *__restrict__ sel,
                                   const int32_t *__restrict__ cnt2d,
                                   const int32_t *__restrict__ first2d,
                                   const int32_t *__restrict__ tboxes,
                                   int32_t *__restrict__ csel, int32_t *__restrict__ fsel,
                                   int32_t *__restrict__ tbsel, int32_t *__restrict__ lsel)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nsel;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t g = sel[k];
        csel[k] = cnt2d[g];
        fsel[k] = first2d[g];
        tbsel[k] = tboxes[g % ntb];
        lsel[k] = (int32_t)(g / ntb);
    }
}

// level boundaries in the selection (lsel ascending): a[l] = first k on
// level >= l, and the entry offset there
__global__ void l3_bounds_kernel(int nl, int64_t nsel, const int32_t *__restrict__ lsel,
                                 const int32_t *__restrict__ starts, int64_t *__restrict__ out)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l > nl) return;
    int64_t lo = 0, hi = nsel;
    while (lo < hi) { const int64_t m = lo + (hi - lo) / 2; if (lsel[m] < l) lo = m + 1; else hi = m; }
    out[l] = lo;
    out[nl + 1 + l] = starts[lo];
}

// each level's CSR starts, [0, c0, c0 + c1, ...], one after the other
__global__ void l3_starts_kernel(int64_t nsel, int nl, const int32_t *__restrict__ lsel,
                                 const int32_t *__restrict__ starts,
                                 const int64_t *__restrict__ bounds, int32_t *__restrict__ out)
{
    const int64_t total = nsel + nl;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (int64_t)gridDim.x * blockDim.x) {
        if (k < nsel) {
            const int l = lsel[k];
            out[k + l] = starts[k] - starts[bounds[l]];
        } else {
            const int l = (int)(k - nsel);   // the closing entry of level l
            const int64_t a = bounds[l], b = bounds[l + 1];
            out[b + l] = starts[b] - starts[a];
        }
    }
}

// List 3 entries of the selection, level after level
__global__ void l3_gather_kernel(int64_t nsel, const int32_t *__restrict__ fsel,
                                 const int32_t *__restrict__ starts,
                                 const int32_t *__restrict__ l3, int32_t *__restrict__ dst)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nsel;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t a = fsel[k];
        for (int32_t j = starts[k]; j < starts[k + 1]; ++j) dst[j] = l3[a + (j - starts[k])];
    }
}

// sort key of a selected (level, target): level, then the target's problem
__global__ void l3_forest_key_kernel(int64_t nsel, int64_t nprob, const int32_t *__restrict__ lsel,
                                     const int32_t *__restrict__ tbsel,
                                     const int32_t *__restrict__ prob, uint64_t *__restrict__ key)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nsel;
         k += (int64_t)gridDim.x * blockDim.x)
        key[k] = (uint64_t)lsel[k] * (uint64_t)nprob + (uint64_t)prob[tbsel[k]];
}

__global__ void permute_kernel(int64_t n, const int32_t *__restrict__ perm,
                               const int32_t *__restrict__ src, int32_t *__restrict__ dst)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        dst[k] = src[perm[k]];
}

__global__ void gather_kernel(int64_t n, const int32_t *__restrict__ idx,
                              const int32_t *__restrict__ src, int32_t *__restrict__ dst)
{
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x)
        dst[k] = src[idx[k]];
}

// }}}

// {{{ small kernels

__global__ void fill_i32_kernel(int64_t n, int32_t v, int32_t *__restrict__ out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = v;
}

__global__ void iota_kernel(int64_t n, int32_t *__restrict__ out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int32_t)i;
}

// tree-order coordinates: out[d * n + i] = x_d[perm[i]]
__global__ void gather_coords_kernel(int64_t n, const int32_t *__restrict__ perm,
                                     const double *__restrict__ x, const double *__restrict__ y,
                                     const double *__restrict__ z, double *__restrict__ out)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = perm[i];
        out[i] = x[u];
        out[n + i] = y[u];
        out[2 * n + i] = z[u];
    }
}

__global__ void inverse_perm_kernel(int64_t n, const int32_t *__restrict__ perm,
                                    int32_t *__restrict__ inv)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        inv[perm[i]] = (int32_t)i;
}

// first position in the sorted box set whose box number is >= level_start[l]
__global__ void set_level_starts_kernel(int nl, const int32_t *__restrict__ level_start,
                                        const int32_t *__restrict__ set, int64_t nset,
                                        int32_t *__restrict__ out)
{
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l > nl) return;
    const int32_t key = level_start[l];
    int64_t lo = 0, hi = nset;
    while (lo < hi) { const int64_t m = lo + (hi - lo) / 2; if (set[m] < key) lo = m + 1; else hi = m; }
    out[l] = (int32_t)lo;
}

// problem of each box: roots are problems 0..P-1, children inherit
__global__ void box_problem_kernel(int32_t b0, int32_t b1, const int32_t *__restrict__ parent,
                                   const int32_t *__restrict__ level, int32_t *__restrict__ prob)
{
    for (int64_t b = b0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < b1;
         b += (int64_t)gridDim.x * blockDim.x)
        prob[b] = level[b] == 0 ? (int32_t)b : prob[parent[b]];
}

// }}}

// {{{ build

struct Arr {
    int kind = 0;        // 0 int32, 1 float64
    int64_t n = 0;
    DevBuf buf;
};

struct State {
    std::map<std::string, Arr> arrays;
};

void put(State &S, const std::string &name, int kind, int64_t n, DevBuf &&buf)
{
    Arr a;
    a.kind = kind;
    a.n = n;
    a.buf = std::move(buf);
    a.buf.st = nullptr;   // released on the legacy default stream
    S.arrays[name] = std::move(a);
}

template <class T>
void put_host(State &S, const std::string &name, const std::vector<T> &v, cudaStream_t st)
{
    DevBuf b = dalloc_n<T>((int64_t)v.size(), st);
    if (!v.empty())
        ck(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st),
           "upload small array");
    // pageable source: the copy is staged before cudaMemcpyAsync returns
    put(S, name, sizeof(T) == 8 ? 1 : 0, (int64_t)v.size(), std::move(b));
}

// indices i < n with flags[i] set, ascending, into out (n entries
// allocated); their number goes to *dcount (device) without waiting
DevBuf select_flagged_async(const uint8_t *flags, int64_t n, int64_t *dcount, cudaStream_t st)
{
    DevBuf out = dalloc_n<int32_t>(std::max<int64_t>(n, 1), st);
    if (n == 0) {
        ck(cudaMemsetAsync(dcount, 0, sizeof(int64_t), st), "memset");
        return out;
    }
    thrust::counting_iterator<int32_t> it(0);
    size_t tmp_bytes = 0;
    ck(cub::DeviceSelect::Flagged(nullptr, tmp_bytes, it, flags, out.as<int32_t>(), dcount, n, st),
       "cub select (size)");
    DevBuf tmp = dalloc(tmp_bytes, st);
    ck(cub::DeviceSelect::Flagged(tmp.p, tmp_bytes, it, flags, out.as<int32_t>(), dcount, n, st),
       "cub select");
    return out;
}

DevBuf select_flagged(const uint8_t *flags, int64_t n, int64_t &count, cudaStream_t st)
{
    DevBuf dn = dalloc_n<int64_t>(1, st);
    DevBuf out = select_flagged_async(flags, n, dn.as<int64_t>(), st);
    count = read_totals(dn, 1, st)[0];
    return out;
}

void copy_d2d(void *dst, const void *src, size_t bytes, cudaStream_t st)
{
    if (bytes) ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st), "copy d2d");
}

void check_err(const DevBuf &err, cudaStream_t st)
{
    int32_t e = 0;
    ck(cudaMemcpyAsync(&e, err.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "copy status");
    ck(cudaStreamSynchronize(st), "list kernels");
    if (e == 1) throw Fail{"a box has more than 27 colleagues (inconsistent tree)"};
    if (e == 2) throw Fail{"List 1/3 traversal stack overflow"};
    if (e == 3) throw Fail{"list counting and filling passes disagree"};
    if (e == 4) throw Fail{"List-2 entry outside the translation classes"};
    if (e) throw Fail{"tree list kernels reported an error"};
}

State *build(int64_t nsrc, const double *sx, const double *sy, const double *sz, int64_t ntgt,
             const double *tx, const double *ty, const double *tz, int32_t nprob,
             const int64_t *src_starts_in, const int64_t *tgt_starts_in, int max_particles,
             int max_levels, const double *bbox_min_in, double root_extent_in, cudaStream_t st)
{
    const bool sat = ntgt < 0 || tx == nullptr;
    if (sat) { ntgt = nsrc; tx = sx; ty = sy; tz = sz; tgt_starts_in = src_starts_in; }
    if (nsrc < 0 || nsrc > INT32_MAX / 2 || ntgt > INT32_MAX / 2) throw Fail{"particle counts out of range"};
    if (max_particles < 1) throw Fail{"max_particles_in_box must be >= 1"};
    if (nprob < 1) throw Fail{"nproblems must be >= 1"};
    if (max_levels < 1 || max_levels > KEY_BITS + 1) max_levels = KEY_BITS + 1;
    std::vector<int64_t> sst(src_starts_in, src_starts_in + nprob + 1);
    std::vector<int64_t> tst(tgt_starts_in, tgt_starts_in + nprob + 1);
    if (sst[0] != 0 || sst[nprob] != nsrc || tst[0] != 0 || tst[nprob] != ntgt)
        throw Fail{"problem starts must run from 0 to the particle count"};
    for (int p = 0; p < nprob; ++p)
        if (sst[p + 1] < sst[p] || tst[p + 1] < tst[p]) throw Fail{"problem starts must not decrease"};
    if (nsrc > 0 && (!sx || !sy || !sz)) throw Fail{"null source coordinates"};

    auto S = std::make_unique<State>();
    // wall time of each phase (each ends with the stream drained)
    std::vector<double> phase_ms;
    auto t_phase = std::chrono::steady_clock::now();
    auto mark = [&]() {
        ck(cudaStreamSynchronize(st), "tree build");
        const auto now = std::chrono::steady_clock::now();
        phase_ms.push_back(std::chrono::duration<double, std::milli>(now - t_phase).count());
        t_phase = now;
    };
    {
        // lexicographic rank of (vx, vy, vz) in [-3,3]^3 \ [-1,1]^3
        int16_t table[343];
        int n = 0;
        for (int a = -3; a <= 3; ++a)
            for (int b = -3; b <= 3; ++b)
                for (int c = -3; c <= 3; ++c) {
                    const int idx = ((a + 3) * 7 + (b + 3)) * 7 + (c + 3);
                    table[idx] = (std::abs(a) <= 1 && std::abs(b) <= 1 && std::abs(c) <= 1)
                                     ? (int16_t)-1 : (int16_t)n++;
                }
        ck(cudaMemcpyToSymbolAsync(c_class_of, table, sizeof(table), 0, cudaMemcpyHostToDevice, st),
           "upload class table");
    }

    // {{{ 1. bounding box

    double lo[3], hi[3];
    {
        constexpr int NPART = 296;   // two blocks per SM per point set
        DevBuf part = dalloc_n<double>(7 * 2 * NPART, st), box = dalloc_n<double>(7, st);
        int nparts = 0;
        if (nsrc > 0) {
            bbox_partial_kernel<<<NPART, 256, 0, st>>>(nsrc, sx, sy, sz, part.as<double>());
            launched("bbox_partial_kernel");
            nparts += NPART;
        }
        if (!sat && ntgt > 0) {
            bbox_partial_kernel<<<NPART, 256, 0, st>>>(ntgt, tx, ty, tz,
                                                       part.as<double>() + 7 * nparts);
            launched("bbox_partial_kernel");
            nparts += NPART;
        }
        double out[7] = {0, 0, 0, 0, 0, 0, 0};
        if (nparts > 0) {
            bbox_combine_kernel<<<1, 256, 0, st>>>(nparts, part.as<double>(), box.as<double>());
            launched("bbox_combine_kernel");
            ck(cudaMemcpyAsync(out, box.p, sizeof(out), cudaMemcpyDeviceToHost, st), "copy bbox");
            ck(cudaStreamSynchronize(st), "bbox");
        }
        if (out[6] > 0) throw Fail{"non-finite particle coordinate"};
        for (int d = 0; d < 3; ++d) { lo[d] = out[d]; hi[d] = out[3 + d]; }
        if (nsrc + (sat ? 0 : ntgt) == 0) for (int d = 0; d < 3; ++d) { lo[d] = 0; hi[d] = 0; }
    }
    double bmin[3], root_extent;
    if (bbox_min_in) {
        if (!(root_extent_in > 0) || !std::isfinite(root_extent_in))
            throw Fail{"root_extent must be positive and finite"};
        for (int d = 0; d < 3; ++d) {
            if (!std::isfinite(bbox_min_in[d])) throw Fail{"non-finite bbox_min"};
            if (nsrc + (sat ? 0 : ntgt) > 0 &&
                (lo[d] < bbox_min_in[d] || hi[d] > bbox_min_in[d] + root_extent_in))
                throw Fail{"a particle lies outside the given root box"};
            bmin[d] = bbox_min_in[d];
        }
        root_extent = root_extent_in;
    } else {
        double ext = 0;
        for (int d = 0; d < 3; ++d) ext = std::max(ext, hi[d] - lo[d]);
        if (ext == 0) ext = 1.0;
        root_extent = ext * (1.0 + 1e-9);
        for (int d = 0; d < 3; ++d) bmin[d] = lo[d] - 0.5 * (root_extent - (hi[d] - lo[d]));
    }

    // }}}

    mark();   // bounding box

    // {{{ 2. keys and sort

    const double scale = (double)(1 << KEY_BITS) / root_extent;
    DevBuf skeys, sperm, tkeys_sorted, tperm;
    {
        DevBuf k = dalloc_n<uint64_t>(nsrc, st), ix = dalloc_n<int32_t>(nsrc, st);
        DevBuf dummy = dalloc_n<unsigned long long>(1, st);
        if (nsrc > 0) {
            keys_kernel<<<std::min<unsigned>(nblocks(nsrc), 148 * 16), 256, 0, st>>>(
                nsrc, sx, sy, sz, bmin[0], bmin[1], bmin[2], scale, root_extent, 0,
                k.as<uint64_t>(), ix.as<int32_t>(), dummy.as<unsigned long long>());
            launched("keys_kernel");
        }
        sort_segments(nsrc, k, ix, sst, st, skeys, sperm);
        if (!sat) {
            DevBuf k2 = dalloc_n<uint64_t>(ntgt, st), ix2 = dalloc_n<int32_t>(ntgt, st);
            if (ntgt > 0) {
                keys_kernel<<<std::min<unsigned>(nblocks(ntgt), 148 * 16), 256, 0, st>>>(
                    ntgt, tx, ty, tz, bmin[0], bmin[1], bmin[2], scale, root_extent, 0,
                    k2.as<uint64_t>(), ix2.as<int32_t>(), dummy.as<unsigned long long>());
                launched("keys_kernel");
            }
            sort_segments(ntgt, k2, ix2, tst, st, tkeys_sorted, tperm);
        }
    }
    const uint64_t *tkeys = sat ? skeys.as<uint64_t>() : tkeys_sorted.as<uint64_t>();

    // }}}

    mark();   // keys and sort

    // {{{ 3. levels

    std::vector<Level> levels;
    levels.emplace_back();
    {
        Level &L0 = levels[0];
        alloc_level(L0, nprob, st);
        std::vector<int32_t> z(nprob, 0), sl(nprob), sh(nprob), tl(nprob), th(nprob), par(nprob, -1);
        for (int p = 0; p < nprob; ++p) {
            sl[p] = (int32_t)sst[p]; sh[p] = (int32_t)sst[p + 1];
            tl[p] = (int32_t)tst[p]; th[p] = (int32_t)tst[p + 1];
        }
        auto up = [&](DevBuf &b, const std::vector<int32_t> &v) {
            ck(cudaMemcpyAsync(b.p, v.data(), 4 * v.size(), cudaMemcpyHostToDevice, st), "upload roots");
        };
        for (int d = 0; d < 3; ++d) up(L0.c[d], z);
        up(L0.slo, sl); up(L0.shi, sh); up(L0.tlo, tl); up(L0.thi, th); up(L0.parent, par);
    }
    std::vector<int32_t> level_start{0};
    for (int l = 0;; ++l) {
        Level &L = levels[l];
        const int32_t base_this = level_start[l];
        if ((int64_t)base_this + L.n > INT32_MAX) throw Fail{"box count exceeds int32"};
        level_start.push_back((int32_t)(base_this + L.n));
        const int allow = (l + 1 < max_levels && l + 1 <= KEY_BITS) ? 1 : 0;
        DevBuf nchild = dalloc_n<int32_t>(L.n, st), bounds = dalloc_n<int32_t>(18 * L.n, st);
        split_count_kernel<<<nblocks(L.n), 256, 0, st>>>(
            L.n, ptrs(L), l, allow, sat ? 1 : 0, max_particles, skeys.as<uint64_t>(), tkeys,
            nchild.as<int32_t>(), bounds.as<int32_t>());
        launched("split_count_kernel");
        DevBuf off;
        const int64_t nnext = scan_counts(nchild.as<int32_t>(), L.n, off, st);
        L.child = dalloc_n<int32_t>(8 * L.n, st);
        Level N;
        alloc_level(N, nnext, st);
        LevelOut o{N.c[0].as<int32_t>(), N.c[1].as<int32_t>(), N.c[2].as<int32_t>(),
                   N.slo.as<int32_t>(), N.shi.as<int32_t>(), N.tlo.as<int32_t>(),
                   N.thi.as<int32_t>(), N.parent.as<int32_t>()};
        split_fill_kernel<<<nblocks(L.n), 256, 0, st>>>(
            L.n, ptrs(L), nchild.as<int32_t>(), bounds.as<int32_t>(), off.as<int32_t>(), nnext,
            base_this, level_start[l + 1], o, L.child.as<int32_t>());
        launched("split_fill_kernel");
        if (nnext == 0) break;
        levels.push_back(std::move(N));
    }
    const int nl = (int)levels.size();
    const int64_t nb = level_start[nl];

    // concatenated box arrays
    DevBuf blev = dalloc_n<int32_t>(nb, st), bc[3], bslo = dalloc_n<int32_t>(nb, st),
           bshi = dalloc_n<int32_t>(nb, st), btlo = dalloc_n<int32_t>(nb, st),
           bthi = dalloc_n<int32_t>(nb, st), bpar = dalloc_n<int32_t>(nb, st),
           bchild = dalloc_n<int32_t>(8 * nb, st), bleaf = dalloc_n<uint8_t>(nb, st);
    for (int d = 0; d < 3; ++d) bc[d] = dalloc_n<int32_t>(nb, st);
    for (int l = 0; l < nl; ++l) {
        const Level &L = levels[l];
        const int64_t o = level_start[l];
        fill_i32_kernel<<<nblocks(L.n), 256, 0, st>>>(L.n, l, blev.as<int32_t>() + o);
        launched("fill_i32_kernel");
        for (int d = 0; d < 3; ++d) copy_d2d(bc[d].as<int32_t>() + o, L.c[d].p, 4 * L.n, st);
        copy_d2d(bslo.as<int32_t>() + o, L.slo.p, 4 * L.n, st);
        copy_d2d(bshi.as<int32_t>() + o, L.shi.p, 4 * L.n, st);
        copy_d2d(btlo.as<int32_t>() + o, L.tlo.p, 4 * L.n, st);
        copy_d2d(bthi.as<int32_t>() + o, L.thi.p, 4 * L.n, st);
        copy_d2d(bpar.as<int32_t>() + o, L.parent.p, 4 * L.n, st);
        copy_d2d(bchild.as<int32_t>() + 8 * o, L.child.p, 32 * L.n, st);
    }
    levels.clear();
    leaf_kernel<<<nblocks(nb), 256, 0, st>>>(nb, bchild.as<int32_t>(), bleaf.as<uint8_t>());
    launched("leaf_kernel");
    BoxPtrs B{blev.as<int32_t>(), bc[0].as<int32_t>(), bc[1].as<int32_t>(), bc[2].as<int32_t>(),
              bslo.as<int32_t>(), bshi.as<int32_t>(), btlo.as<int32_t>(), bthi.as<int32_t>(),
              bpar.as<int32_t>(), bchild.as<int32_t>(), bleaf.as<uint8_t>(), nb};
    DevBuf recs = dalloc_n<Rec>(nb, st);
    pack_records_kernel<<<nblocks(nb), 256, 0, st>>>(B, recs.as<Rec>());
    launched("pack_records_kernel");
    const Rec *R = recs.as<Rec>();

    // }}}

    mark();   // levels

    // {{{ 4. box attributes, box sets, colleagues

    {
        DevBuf centers = dalloc_n<double>(3 * nb, st), olev = dalloc_n<int32_t>(nb, st),
               opar = dalloc_n<int32_t>(nb, st), ochild = dalloc_n<int32_t>(8 * nb, st),
               ocoords = dalloc_n<int32_t>(3 * nb, st), sstart = dalloc_n<int32_t>(nb, st),
               scum = dalloc_n<int32_t>(nb, st), snc = dalloc_n<int32_t>(nb, st),
               tstart = dalloc_n<int32_t>(nb, st), tcum = dalloc_n<int32_t>(nb, st),
               tnc = dalloc_n<int32_t>(nb, st);
        DevBuf f_src = dalloc_n<uint8_t>(nb, st), f_tgt = dalloc_n<uint8_t>(nb, st),
               f_sp = dalloc_n<uint8_t>(nb, st), f_ttp = dalloc_n<uint8_t>(nb, st);
        attrs_kernel<<<nblocks(nb), 256, 0, st>>>(
            B, bmin[0], bmin[1], bmin[2], root_extent, centers.as<double>(), olev.as<int32_t>(),
            opar.as<int32_t>(), ochild.as<int32_t>(), ocoords.as<int32_t>(),
            sstart.as<int32_t>(), scum.as<int32_t>(), snc.as<int32_t>(), tstart.as<int32_t>(),
            tcum.as<int32_t>(), tnc.as<int32_t>(), f_src.as<uint8_t>(), f_tgt.as<uint8_t>(),
            f_sp.as<uint8_t>(), f_ttp.as<uint8_t>());
        launched("attrs_kernel");
        put(*S, "box_centers", 1, 3 * nb, std::move(centers));
        put(*S, "box_levels", 0, nb, std::move(olev));
        put(*S, "box_parent_ids", 0, nb, std::move(opar));
        put(*S, "box_child_ids", 0, 8 * nb, std::move(ochild));
        put(*S, "box_coords", 0, 3 * nb, std::move(ocoords));
        put(*S, "box_source_starts", 0, nb, std::move(sstart));
        put(*S, "box_source_counts_cumul", 0, nb, std::move(scum));
        put(*S, "box_source_counts_nonchild", 0, nb, std::move(snc));
        put(*S, "box_target_starts", 0, nb, std::move(tstart));
        put(*S, "box_target_counts_cumul", 0, nb, std::move(tcum));
        put(*S, "box_target_counts_nonchild", 0, nb, std::move(tnc));

        DevBuf dls = dalloc_n<int32_t>(nl + 1, st);
        ck(cudaMemcpyAsync(dls.p, level_start.data(), 4 * (nl + 1), cudaMemcpyHostToDevice, st),
           "upload level starts");
        const char *names[4] = {"source_boxes", "target_boxes", "source_parent_boxes",
                                "target_or_target_parent_boxes"};
        const char *lsnames[4] = {"level_start_source_box_nrs", "level_start_target_box_nrs",
                                  "level_start_source_parent_box_nrs",
                                  "level_start_target_or_target_parent_box_nrs"};
        const DevBuf *flags[4] = {&f_src, &f_tgt, &f_sp, &f_ttp};
        DevBuf dcnt = dalloc_n<int64_t>(4, st);
        DevBuf sets[4];
        for (int k = 0; k < 4; ++k)
            sets[k] = select_flagged_async(flags[k]->as<uint8_t>(), nb, dcnt.as<int64_t>() + k, st);
        const std::vector<int64_t> cnt = read_totals(dcnt, 4, st);
        for (int k = 0; k < 4; ++k) {
            DevBuf ls = dalloc_n<int32_t>(nl + 1, st);
            set_level_starts_kernel<<<1, 64 * ((nl + 64) / 64), 0, st>>>(
                nl, dls.as<int32_t>(), sets[k].as<int32_t>(), cnt[k], ls.as<int32_t>());
            launched("set_level_starts_kernel");
            put(*S, names[k], 0, cnt[k], std::move(sets[k]));
            put(*S, lsnames[k], 0, nl + 1, std::move(ls));
        }
        put(*S, "level_start_box_nrs", 0, nl + 1, std::move(dls));

        DevBuf prob = dalloc_n<int32_t>(nb, st);
        for (int l = 0; l < nl; ++l) {
            box_problem_kernel<<<nblocks(level_start[l + 1] - level_start[l]), 256, 0, st>>>(
                level_start[l], level_start[l + 1], bpar.as<int32_t>(), blev.as<int32_t>(),
                prob.as<int32_t>());
            launched("box_problem_kernel");
        }
        put(*S, "box_problem", 0, nb, std::move(prob));
    }

    DevBuf coll = dalloc_n<int32_t>(MAXCOLL * nb, st), ncoll = dalloc_n<int32_t>(nb, st);
    DevBuf err = dalloc_n<int32_t>(1, st);
    ck(cudaMemsetAsync(err.p, 0, 4, st), "memset");
    for (int l = 0; l < nl; ++l) {
        colleagues_kernel<<<nblocks(level_start[l + 1] - level_start[l]), 256, 0, st>>>(
            R, level_start[l], level_start[l + 1], coll.as<int32_t>(), ncoll.as<int32_t>(),
            err.as<int32_t>());
        launched("colleagues_kernel");
    }

    // }}}

    mark();   // boxes, sets, colleagues

    // {{{ 5. lists

    const Arr &TB = S->arrays.at("target_boxes");
    const Arr &TTP = S->arrays.at("target_or_target_parent_boxes");
    const int64_t ntb = TB.n, nttp = TTP.n;
    DevBuf n1 = dalloc_n<int32_t>(ntb, st), n3 = dalloc_n<int32_t>(ntb, st);
    lists13_kernel<<<nblocks(ntb, 128), 128, 0, st>>>(
        R, coll.as<int32_t>(), ncoll.as<int32_t>(), ntb, TB.buf.as<int32_t>(), 0,
        n1.as<int32_t>(), n3.as<int32_t>(), nullptr, nullptr, nullptr, nullptr, err.as<int32_t>());
    launched("lists13_kernel");
    DevBuf n2 = dalloc_n<int32_t>(nttp, st), n4 = dalloc_n<int32_t>(nttp, st);
    lists24_kernel<<<nblocks(nttp, 128), 128, 0, st>>>(
        R, coll.as<int32_t>(), ncoll.as<int32_t>(), nttp, TTP.buf.as<int32_t>(), 0,
        n2.as<int32_t>(), n4.as<int32_t>(), nullptr, nullptr, nullptr, nullptr, nullptr,
        err.as<int32_t>());
    launched("lists24_kernel");
    DevBuf s1, s2, s3, s4;
    DevBuf dtot = dalloc_n<int64_t>(4, st);
    scan_counts_async(n1.as<int32_t>(), ntb, s1, dtot.as<int64_t>() + 0, st);
    scan_counts_async(n2.as<int32_t>(), nttp, s2, dtot.as<int64_t>() + 1, st);
    scan_counts_async(n3.as<int32_t>(), ntb, s3, dtot.as<int64_t>() + 2, st);
    scan_counts_async(n4.as<int32_t>(), nttp, s4, dtot.as<int64_t>() + 3, st);
    const std::vector<int64_t> tot = read_totals(dtot, 4, st);
    const int64_t t1 = tot[0], t2 = tot[1], t3 = tot[2], t4 = tot[3];
    DevBuf l1 = dalloc_n<int32_t>(t1, st), l3 = dalloc_n<int32_t>(t3, st);
    lists13_kernel<<<nblocks(ntb, 128), 128, 0, st>>>(
        R, coll.as<int32_t>(), ncoll.as<int32_t>(), ntb, TB.buf.as<int32_t>(), 1, nullptr,
        nullptr, s1.as<int32_t>(), s3.as<int32_t>(), l1.as<int32_t>(), l3.as<int32_t>(),
        err.as<int32_t>());
    launched("lists13_kernel");

    DevBuf l2 = dalloc_n<int32_t>(t2, st), l2c = dalloc_n<int32_t>(t2, st),
           l4 = dalloc_n<int32_t>(t4, st);
    lists24_kernel<<<nblocks(nttp, 128), 128, 0, st>>>(
        R, coll.as<int32_t>(), ncoll.as<int32_t>(), nttp, TTP.buf.as<int32_t>(), 1, nullptr,
        nullptr, s2.as<int32_t>(), s4.as<int32_t>(), l2.as<int32_t>(), l2c.as<int32_t>(),
        l4.as<int32_t>(), err.as<int32_t>());
    launched("lists24_kernel");
    check_err(err, st);

    mark();   // lists 1-4

    // List 3 by source level: all (level, target) pairs in one pass
    {
        const int64_t n2d = (int64_t)nl * ntb;
        DevBuf first2d = dalloc_n<int32_t>(n2d, st), cnt2d = dalloc_n<int32_t>(n2d, st);
        DevBuf flag2d = dalloc_n<uint8_t>(n2d, st);
        DevBuf dls = dalloc_n<int32_t>(nl + 1, st);
        ck(cudaMemcpyAsync(dls.p, level_start.data(), 4 * (nl + 1), cudaMemcpyHostToDevice, st),
           "upload level starts");
        int64_t nsel = 0;
        DevBuf sel;
        if (ntb > 0) {
            l3_levels_kernel<<<nblocks(ntb), 256, 0, st>>>(ntb, nl, s3.as<int32_t>(),
                                                           l3.as<int32_t>(), dls.as<int32_t>(),
                                                           first2d.as<int32_t>(),
                                                           cnt2d.as<int32_t>(), flag2d.as<uint8_t>());
            launched("l3_levels_kernel");
            sel = select_flagged(flag2d.as<uint8_t>(), n2d, nsel, st);
        }
        DevBuf csel = dalloc_n<int32_t>(nsel, st), fsel = dalloc_n<int32_t>(nsel, st),
               tbsel = dalloc_n<int32_t>(nsel, st), lsel = dalloc_n<int32_t>(nsel, st);
        if (nsel > 0) {
            l3_selected_kernel<<<nblocks(nsel), 256, 0, st>>>(
                nsel, ntb, sel.as<int32_t>(), cnt2d.as<int32_t>(), first2d.as<int32_t>(),
                TB.buf.as<int32_t>(), csel.as<int32_t>(), fsel.as<int32_t>(),
                tbsel.as<int32_t>(), lsel.as<int32_t>());
            launched("l3_selected_kernel");
        }
        if (nprob > 1 && nsel > 1) {
            // a forest lists one level's targets problem after problem (target
            // level, then Morton, inside a problem): stable sort by (level, problem)
            DevBuf key = dalloc_n<uint64_t>(nsel, st), key2 = dalloc_n<uint64_t>(nsel, st);
            DevBuf iota = dalloc_n<int32_t>(nsel, st), perm = dalloc_n<int32_t>(nsel, st);
            l3_forest_key_kernel<<<nblocks(nsel), 256, 0, st>>>(
                nsel, nprob, lsel.as<int32_t>(), tbsel.as<int32_t>(),
                S->arrays.at("box_problem").buf.as<int32_t>(), key.as<uint64_t>());
            launched("l3_forest_key_kernel");
            iota_kernel<<<nblocks(nsel), 256, 0, st>>>(nsel, iota.as<int32_t>());
            launched("iota_kernel");
            size_t tmp_bytes = 0;
            ck(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.as<uint64_t>(),
                                               key2.as<uint64_t>(), iota.as<int32_t>(),
                                               perm.as<int32_t>(), (int)nsel, 0, 64, st),
               "cub sort (size)");
            DevBuf tmp = dalloc(tmp_bytes, st);
            ck(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, key.as<uint64_t>(),
                                               key2.as<uint64_t>(), iota.as<int32_t>(),
                                               perm.as<int32_t>(), (int)nsel, 0, 64, st),
               "cub sort");
            DevBuf *cols[4] = {&csel, &fsel, &tbsel, &lsel};
            for (DevBuf *c : cols) {
                DevBuf out = dalloc_n<int32_t>(nsel, st);
                permute_kernel<<<nblocks(nsel), 256, 0, st>>>(nsel, perm.as<int32_t>(),
                                                              c->as<int32_t>(), out.as<int32_t>());
                launched("permute_kernel");
                *c = std::move(out);
            }
        }
        DevBuf starts;
        const int64_t nent = scan_counts(csel.as<int32_t>(), nsel, starts, st);
        DevBuf li_all = dalloc_n<int32_t>(nent, st);
        DevBuf bounds = dalloc_n<int64_t>(2 * (nl + 1), st);
        DevBuf st_all = dalloc_n<int32_t>(nsel + nl, st);
        l3_bounds_kernel<<<1, 64 * ((nl + 64) / 64), 0, st>>>(nl, nsel, lsel.as<int32_t>(),
                                                              starts.as<int32_t>(),
                                                              bounds.as<int64_t>());
        launched("l3_bounds_kernel");
        if (nsel > 0) {
            l3_gather_kernel<<<nblocks(nsel), 256, 0, st>>>(nsel, fsel.as<int32_t>(),
                                                            starts.as<int32_t>(), l3.as<int32_t>(),
                                                            li_all.as<int32_t>());
            launched("l3_gather_kernel");
        }
        l3_starts_kernel<<<nblocks(nsel + nl), 256, 0, st>>>(nsel, nl, lsel.as<int32_t>(),
                                                            starts.as<int32_t>(),
                                                            bounds.as<int64_t>(),
                                                            st_all.as<int32_t>());
        launched("l3_starts_kernel");
        std::vector<int64_t> hb(2 * (nl + 1));
        ck(cudaMemcpyAsync(hb.data(), bounds.p, 8 * hb.size(), cudaMemcpyDeviceToHost, st),
           "copy level bounds");
        ck(cudaStreamSynchronize(st), "list 3 by level");
        std::vector<int32_t> tbls(nl + 1), stoff(nl + 1), lioff(nl + 1);
        for (int l = 0; l <= nl; ++l) {
            tbls[l] = (int32_t)hb[l];
            stoff[l] = (int32_t)(hb[l] + l);
            lioff[l] = (int32_t)hb[nl + 1 + l];
        }
        put(*S, "sep_smaller_target_boxes", 0, nsel, std::move(tbsel));
        put_host(*S, "sep_smaller_target_boxes_level_starts", tbls, st);
        put(*S, "sep_smaller_starts", 0, nsel + nl, std::move(st_all));
        put_host(*S, "sep_smaller_starts_level_offsets", stoff, st);
        put(*S, "sep_smaller_lists", 0, nent, std::move(li_all));
        put_host(*S, "sep_smaller_lists_level_offsets", lioff, st);
    }
    put(*S, "neighbor_source_boxes_starts", 0, ntb + 1, std::move(s1));
    put(*S, "neighbor_source_boxes_lists", 0, t1, std::move(l1));
    put(*S, "from_sep_siblings_starts", 0, nttp + 1, std::move(s2));
    put(*S, "from_sep_siblings_lists", 0, t2, std::move(l2));
    put(*S, "from_sep_siblings_translation_classes", 0, t2, std::move(l2c));
    put(*S, "from_sep_bigger_starts", 0, nttp + 1, std::move(s4));
    put(*S, "from_sep_bigger_lists", 0, t4, std::move(l4));

    // }}}

    mark();   // list 3 by level

    // {{{ 6. particles, translation classes, scalars

    {
        DevBuf srt = dalloc_n<double>(3 * nsrc, st);
        if (nsrc > 0) {
            gather_coords_kernel<<<nblocks(nsrc), 256, 0, st>>>(nsrc, sperm.as<int32_t>(), sx, sy,
                                                                sz, srt.as<double>());
            launched("gather_coords_kernel");
        }
        const DevBuf &tp = sat ? sperm : tperm;
        DevBuf trt = dalloc_n<double>(3 * ntgt, st), sti = dalloc_n<int32_t>(ntgt, st);
        if (ntgt > 0) {
            gather_coords_kernel<<<nblocks(ntgt), 256, 0, st>>>(ntgt, tp.as<int32_t>(), tx, ty,
                                                                tz, trt.as<double>());
            launched("gather_coords_kernel");
            inverse_perm_kernel<<<nblocks(ntgt), 256, 0, st>>>(ntgt, tp.as<int32_t>(),
                                                               sti.as<int32_t>());
            launched("inverse_perm_kernel");
        }
        put(*S, "sources", 1, 3 * nsrc, std::move(srt));
        put(*S, "targets", 1, 3 * ntgt, std::move(trt));
        put(*S, "sorted_target_ids", 0, ntgt, std::move(sti));
        if (sat) {
            DevBuf tts = dalloc_n<int32_t>(nsrc, st);
            if (nsrc > 0) {
                iota_kernel<<<nblocks(nsrc), 256, 0, st>>>(nsrc, tts.as<int32_t>());
                launched("iota_kernel");
            }
            put(*S, "target_to_source", 0, nsrc, std::move(tts));
        }
        put(*S, "user_source_ids", 0, nsrc, std::move(sperm));
    }
    {
        std::vector<int32_t> cls_ls(nl + 1, 0);
        for (int l = 0; l < nl; ++l) cls_ls[l + 1] = cls_ls[l] + (l >= 2 ? NCLASSES : 0);
        const int64_t ncl = cls_ls[nl];
        std::vector<double> cvec(3 * (size_t)ncl);
        for (int l = 2; l < nl; ++l) {
            const double h = root_extent / (double)(1LL << l);
            int k = 0;
            for (int a = -3; a <= 3; ++a)
                for (int b2 = -3; b2 <= 3; ++b2)
                    for (int c = -3; c <= 3; ++c) {
                        if (std::abs(a) <= 1 && std::abs(b2) <= 1 && std::abs(c) <= 1) continue;
                        const int64_t g = cls_ls[l] + k++;
                        cvec[g] = a * h; cvec[ncl + g] = b2 * h; cvec[2 * ncl + g] = c * h;
                    }
        }
        put_host(*S, "from_sep_siblings_translation_classes_level_starts", cls_ls, st);
        put_host(*S, "from_sep_siblings_translation_class_to_distance_vector", cvec, st);
        put_host(*S, "bbox_min", std::vector<double>(bmin, bmin + 3), st);
        put_host(*S, "root_extent", std::vector<double>(1, root_extent), st);
        put_host(*S, "scalars", std::vector<int32_t>{(int32_t)nb, nl, (int32_t)nsrc,
                                                     (int32_t)ntgt, sat ? 1 : 0}, st);
    }
    mark();   // particles, classes, scalars
    put_host(*S, "build_phase_ms", phase_ms, st);
    ck(cudaStreamSynchronize(st), "tree build");
    return S.release();

    // }}}
}

// }}}

}  // namespace gtree
}  // namespace sumpy

using namespace sumpy;

extern "C" {

int sumpy_tree_gpu_build(int64_t nsources, const double *sx, const double *sy, const double *sz,
                         int64_t ntargets, const double *tx, const double *ty, const double *tz,
                         int32_t nproblems, const int64_t *problem_source_starts,
                         const int64_t *problem_target_starts, int max_particles_in_box,
                         int max_levels, const double *bbox_min, double root_extent,
                         void *stream, void **handle_out)
{
    if (!handle_out) return bad_arg("tree_gpu: handle_out is NULL");
    *handle_out = nullptr;
    int64_t one[2] = {0, nsources};
    int64_t onet[2] = {0, ntargets};
    if (nproblems < 1) return bad_arg("tree_gpu: nproblems must be >= 1");
    if (nproblems > 1 && !problem_source_starts)
        return bad_arg("tree_gpu: a forest needs problem_source_starts");
    const bool sat = ntargets < 0 || tx == nullptr;
    if (nproblems > 1 && !sat && !problem_target_starts)
        return bad_arg("tree_gpu: a forest with targets needs problem_target_starts");
    try {
        *handle_out = gtree::build(nsources, sx, sy, sz, ntargets, tx, ty, tz, nproblems,
                                   nproblems > 1 ? problem_source_starts : one,
                                   nproblems > 1 ? problem_target_starts : onet,
                                   max_particles_in_box, max_levels, bbox_min, root_extent,
                                   as_stream(stream));
        return SUMPY_OK;
    } catch (const gtree::Fail &f) {
        set_last_error("tree_gpu: " + f.msg);
        return SUMPY_EINVAL;
    } catch (const std::exception &e) {
        set_last_error(std::string("tree_gpu: ") + e.what());
        return SUMPY_ELAUNCH;
    }
}

int sumpy_tree_gpu_array_info(void *handle, const char *name, int *kind, int64_t *length)
{
    auto *S = static_cast<gtree::State *>(handle);
    if (!S || !name || !kind || !length) return bad_arg("tree_gpu: null argument");
    auto it = S->arrays.find(name);
    if (it == S->arrays.end()) {
        set_last_error(std::string("tree_gpu: no array ") + name);
        return SUMPY_EINVAL;
    }
    *kind = it->second.kind;
    *length = it->second.n;
    return SUMPY_OK;
}

int sumpy_tree_gpu_array_copy(void *handle, const char *name, void *dst, int64_t capacity_bytes,
                              int dst_on_device, void *stream)
{
    auto *S = static_cast<gtree::State *>(handle);
    if (!S || !name) return bad_arg("tree_gpu: null argument");
    auto it = S->arrays.find(name);
    if (it == S->arrays.end()) {
        set_last_error(std::string("tree_gpu: no array ") + name);
        return SUMPY_EINVAL;
    }
    const gtree::Arr &a = it->second;
    const size_t bytes = (size_t)a.n * (a.kind == 0 ? 4 : 8);
    if ((int64_t)bytes > capacity_bytes) return bad_arg("tree_gpu: destination too small");
    if (!bytes) return SUMPY_OK;
    if (!dst) return bad_arg("tree_gpu: null destination");
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaMemcpyAsync(dst, a.buf.p, bytes,
                                    dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    st);
    if (e == cudaSuccess && !dst_on_device) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_last_error(std::string("tree_gpu: copy: ") + cudaGetErrorString(e));
        return SUMPY_ELAUNCH;
    }
    return SUMPY_OK;
}

void sumpy_tree_gpu_free(void *handle) { delete static_cast<gtree::State *>(handle); }

}  // extern "C"
