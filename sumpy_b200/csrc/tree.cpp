// Octree, FMM interaction lists and translation classes for 3D point sets.
//
// This is the stand-in for boxtree (TreeBuilder, FMMTraversalBuilder,
// TranslationClassesBuilder), which sumpy depends on (sumpy/fmm.py:356-363)
// but which is not part of the sumpy sources. It produces the arrays, under
// boxtree's names, that sumpy's expansion wrangler consumes (sumpy/fmm.py:
// 372-397, 543-592, 609-1083): tree-order particles, level-ordered boxes,
// and the four interaction lists of the adaptive FMM with one-box
// separation (well_sep_is_n_away = 1).
//
// Tree: a box is refined while it holds more than max_particles_in_box
// particles (sources + targets, or sources only when sources are the
// targets); empty children are not created. Boxes are numbered level by
// level, in Morton order within a level. Particles are sorted by Morton key
// so every box owns a contiguous range.
//
// Lists (t = target box, s = source box; "adjacent" = closed boxes touch):
//   List 1  leaf t with targets: leaf boxes with sources adjacent to t.
//   List 2  t with targets below it, level >= 2: boxes with sources that are
//           children of a colleague of parent(t) and not adjacent to t.
//   List 3  leaf t with targets: boxes with sources below a colleague of t,
//           not adjacent to t, whose parent is adjacent to t.
//   List 4  t with targets below it: leaf boxes with sources on a level
//           coarser than t, adjacent to parent(t), not adjacent to t.
// Every (target, source) pair is covered exactly once by List 1, List 3, or
// an ancestor-or-self of the target through List 2 or List 4.
//
// Translation classes: per level >= 2 the 316 vectors v in [-3,3]^3 minus
// [-1,1]^3 (target center - source center in box widths), enumerated in
// lexicographic order of (vx, vy, vz).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/sumpy_b200_tree.h"

namespace {

constexpr int KEY_BITS = 21;

struct Array {
    int kind;  // 0 = int32, 1 = float64
    std::vector<int32_t> i;
    std::vector<double> d;
};

struct TreeState {
    std::map<std::string, Array> arrays;
    std::string error;

    void put_i(const std::string &name, std::vector<int32_t> v)
    {
        Array a; a.kind = 0; a.i = std::move(v); arrays[name] = std::move(a);
    }
    void put_d(const std::string &name, std::vector<double> v)
    {
        Array a; a.kind = 1; a.d = std::move(v); arrays[name] = std::move(a);
    }
};

thread_local std::string g_last_error;

inline uint64_t spread3(uint32_t v)
{
    uint64_t x = v & 0x1fffff;
    x = (x | (x << 32)) & 0x1f00000000ffffULL;
    x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

struct Box {
    int level;
    int32_t c[3];       // integer coords at own level
    int64_t s_lo, s_hi; // sorted source range
    int64_t t_lo, t_hi; // sorted target range
    int32_t parent;
    int octant;
};

struct Builder {
    // inputs
    int64_t nsrc, ntgt;
    bool sources_are_targets;
    int max_particles, max_levels;

    double bbox_min[3], root_extent;
    std::vector<uint64_t> skey, tkey;
    std::vector<int32_t> sperm, tperm;

    std::vector<Box> boxes;
    std::vector<int32_t> level_start;
    std::vector<int32_t> children;  // [nboxes][8], -1 if none (internal)
    int nlevels = 0;

    int64_t lo_fine(int32_t b, int d) const
    {
        return (int64_t)boxes[b].c[d] << (KEY_BITS - boxes[b].level);
    }
    int64_t hi_fine(int32_t b, int d) const
    {
        return ((int64_t)boxes[b].c[d] + 1) << (KEY_BITS - boxes[b].level);
    }
    bool adjacent(int32_t a, int32_t b) const
    {
        for (int d = 0; d < 3; ++d)
            if (lo_fine(a, d) > hi_fine(b, d) || lo_fine(b, d) > hi_fine(a, d)) return false;
        return true;
    }
    bool is_leaf(int32_t b) const
    {
        for (int o = 0; o < 8; ++o) if (children[8 * (size_t)b + o] >= 0) return false;
        return true;
    }
    bool has_sources(int32_t b) const { return boxes[b].s_hi > boxes[b].s_lo; }
    bool has_targets(int32_t b) const { return boxes[b].t_hi > boxes[b].t_lo; }
};

void compute_keys(const double *x, const double *y, const double *z, int64_t n,
                  const double *bmin, double extent, std::vector<uint64_t> &keys)
{
    keys.resize(n);
    const double scale = (double)(1 << KEY_BITS) / extent;
    const uint32_t maxc = (1u << KEY_BITS) - 1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double p[3] = {x[i], y[i], z[i]};
        uint32_t q[3];
        for (int d = 0; d < 3; ++d) {
            double v = std::floor((p[d] - bmin[d]) * scale);
            if (v < 0) v = 0;
            if (v > maxc) v = maxc;
            q[d] = (uint32_t)v;
        }
        keys[i] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    }
}

void sort_by_key(const std::vector<uint64_t> &keys, std::vector<int32_t> &perm)
{
    perm.resize(keys.size());
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(),
                     [&](int32_t a, int32_t b) { return keys[a] < keys[b]; });
}

inline int octant_of(uint64_t key, int child_level)
{
    return (int)((key >> (3 * (KEY_BITS - child_level))) & 7);
}

// first index in [lo, hi) whose octant at child_level is >= oct
int64_t octant_bound(const std::vector<uint64_t> &sorted_keys, int64_t lo, int64_t hi,
                     int child_level, int oct)
{
    while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if (octant_of(sorted_keys[mid], child_level) < oct) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

void build_tree(Builder &B)
{
    std::vector<uint64_t> sk(B.nsrc), tk(B.ntgt);
    for (int64_t i = 0; i < B.nsrc; ++i) sk[i] = B.skey[B.sperm[i]];
    if (!B.sources_are_targets)
        for (int64_t i = 0; i < B.ntgt; ++i) tk[i] = B.tkey[B.tperm[i]];
    const std::vector<uint64_t> &tkeys = B.sources_are_targets ? sk : tk;

    Box root{};
    root.level = 0; root.c[0] = root.c[1] = root.c[2] = 0;
    root.s_lo = 0; root.s_hi = B.nsrc; root.t_lo = 0; root.t_hi = B.ntgt;
    root.parent = -1; root.octant = 0;
    B.boxes.push_back(root);
    B.level_start.push_back(0);
    size_t lev_begin = 0, lev_end = 1;
    int level = 0;
    while (true) {
        B.children.resize(8 * B.boxes.size(), -1);
        std::vector<Box> next;
        for (size_t bi = lev_begin; bi < lev_end; ++bi) {
            const Box &b = B.boxes[bi];
            int64_t count = (b.s_hi - b.s_lo) + (B.sources_are_targets ? 0 : (b.t_hi - b.t_lo));
            if (count <= B.max_particles || level + 1 >= B.max_levels || level + 1 > KEY_BITS)
                continue;
            int64_t sb[9], tb[9];
            sb[0] = b.s_lo; sb[8] = b.s_hi; tb[0] = b.t_lo; tb[8] = b.t_hi;
            for (int o = 1; o < 8; ++o) {
                sb[o] = octant_bound(sk, b.s_lo, b.s_hi, level + 1, o);
                tb[o] = octant_bound(tkeys, b.t_lo, b.t_hi, level + 1, o);
            }
            for (int o = 0; o < 8; ++o) {
                if (sb[o + 1] == sb[o] && tb[o + 1] == tb[o]) continue;
                Box c{};
                c.level = level + 1;
                c.c[0] = 2 * b.c[0] + ((o >> 2) & 1);
                c.c[1] = 2 * b.c[1] + ((o >> 1) & 1);
                c.c[2] = 2 * b.c[2] + (o & 1);
                c.s_lo = sb[o]; c.s_hi = sb[o + 1]; c.t_lo = tb[o]; c.t_hi = tb[o + 1];
                c.parent = (int32_t)bi; c.octant = o;
                B.children[8 * bi + o] = (int32_t)(B.boxes.size() + next.size());
                next.push_back(c);
            }
        }
        if (next.empty()) break;
        lev_begin = B.boxes.size();
        B.level_start.push_back((int32_t)lev_begin);
        B.boxes.insert(B.boxes.end(), next.begin(), next.end());
        lev_end = B.boxes.size();
        ++level;
    }
    B.children.resize(8 * B.boxes.size(), -1);
    B.level_start.push_back((int32_t)B.boxes.size());
    B.nlevels = (int)B.level_start.size() - 1;
}

inline int class_of(int vx, int vy, int vz)
{
    // lexicographic rank of (vx, vy, vz) in [-3,3]^3 \ [-1,1]^3
    static int table[343];
    static bool init = false;
    if (!init) {
        int n = 0;
        for (int a = -3; a <= 3; ++a)
            for (int b = -3; b <= 3; ++b)
                for (int c = -3; c <= 3; ++c) {
                    int idx = ((a + 3) * 7 + (b + 3)) * 7 + (c + 3);
                    if (std::abs(a) <= 1 && std::abs(b) <= 1 && std::abs(c) <= 1) table[idx] = -1;
                    else table[idx] = n++;
                }
        init = true;
    }
    if (vx < -3 || vx > 3 || vy < -3 || vy > 3 || vz < -3 || vz > 3) return -1;
    return table[((vx + 3) * 7 + (vy + 3)) * 7 + (vz + 3)];
}

constexpr int NCLASSES = 316;

void to_csr(const std::vector<std::vector<int32_t>> &lists, std::vector<int32_t> &starts,
            std::vector<int32_t> &flat)
{
    starts.assign(lists.size() + 1, 0);
    for (size_t i = 0; i < lists.size(); ++i) starts[i + 1] = starts[i] + (int32_t)lists[i].size();
    flat.resize(starts.back());
    for (size_t i = 0; i < lists.size(); ++i)
        std::copy(lists[i].begin(), lists[i].end(), flat.begin() + starts[i]);
}

}  // namespace

extern "C" {

const char *sumpy_tree_last_error(void) { return g_last_error.c_str(); }

int sumpy_tree_build(int64_t nsources, const double *sx, const double *sy, const double *sz,
                     int64_t ntargets, const double *tx, const double *ty, const double *tz,
                     int max_particles_in_box, int max_levels, void **handle_out)
{
    return sumpy_tree_build_in_box(nsources, sx, sy, sz, ntargets, tx, ty, tz,
                                   max_particles_in_box, max_levels, nullptr, 0.0, handle_out);
}

int sumpy_tree_build_in_box(int64_t nsources, const double *sx, const double *sy,
                            const double *sz, int64_t ntargets, const double *tx,
                            const double *ty, const double *tz, int max_particles_in_box,
                            int max_levels, const double *bbox_min, double root_extent,
                            void **handle_out)
{
    try {
        if (!handle_out) { g_last_error = "handle_out is NULL"; return SUMPY_TREE_EINVAL; }
        *handle_out = nullptr;
        if (nsources < 0 || nsources > INT32_MAX / 2 || ntargets > INT32_MAX / 2) {
            g_last_error = "particle counts out of range"; return SUMPY_TREE_EINVAL;
        }
        if (max_particles_in_box < 1) {
            g_last_error = "max_particles_in_box must be >= 1"; return SUMPY_TREE_EINVAL;
        }
        if (max_levels < 1 || max_levels > KEY_BITS + 1) max_levels = KEY_BITS + 1;
        const bool sat = (ntargets < 0) || (tx == nullptr);
        if (sat) { ntargets = nsources; tx = sx; ty = sy; tz = sz; }

        Builder B;
        B.nsrc = nsources; B.ntgt = ntargets; B.sources_are_targets = sat;
        B.max_particles = max_particles_in_box; B.max_levels = max_levels;

        double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        auto upd = [&](const double *x, const double *y, const double *z, int64_t n) {
            for (int64_t i = 0; i < n; ++i) {
                const double p[3] = {x[i], y[i], z[i]};
                for (int d = 0; d < 3; ++d) {
                    if (!std::isfinite(p[d])) throw std::string("non-finite particle coordinate");
                    lo[d] = std::min(lo[d], p[d]); hi[d] = std::max(hi[d], p[d]);
                }
            }
        };
        upd(sx, sy, sz, nsources);
        if (!sat) upd(tx, ty, tz, ntargets);
        if (nsources + (sat ? 0 : ntargets) == 0) { for (int d = 0; d < 3; ++d) { lo[d] = 0; hi[d] = 0; } }
        if (bbox_min) {
            // caller-fixed root box (trees of a batch share their level geometry)
            if (!(root_extent > 0) || !std::isfinite(root_extent))
                throw std::string("root_extent must be positive and finite");
            for (int d = 0; d < 3; ++d) {
                if (!std::isfinite(bbox_min[d])) throw std::string("non-finite bbox_min");
                if (nsources + (sat ? 0 : ntargets) > 0 &&
                    (lo[d] < bbox_min[d] || hi[d] > bbox_min[d] + root_extent))
                    throw std::string("a particle lies outside the given root box");
                B.bbox_min[d] = bbox_min[d];
            }
            B.root_extent = root_extent;
        } else {
            double ext = 0;
            for (int d = 0; d < 3; ++d) ext = std::max(ext, hi[d] - lo[d]);
            if (ext == 0) ext = 1.0;
            // enlarge slightly so that the maximal coordinates fall inside the root box
            B.root_extent = ext * (1.0 + 1e-9);
            for (int d = 0; d < 3; ++d)
                B.bbox_min[d] = lo[d] - 0.5 * (B.root_extent - (hi[d] - lo[d]));
        }

        compute_keys(sx, sy, sz, nsources, B.bbox_min, B.root_extent, B.skey);
        sort_by_key(B.skey, B.sperm);
        if (!sat) {
            compute_keys(tx, ty, tz, ntargets, B.bbox_min, B.root_extent, B.tkey);
            sort_by_key(B.tkey, B.tperm);
        }
        build_tree(B);

        auto *S = new TreeState();
        const int64_t nb = (int64_t)B.boxes.size();
        const int nl = B.nlevels;

        // {{{ tree arrays

        std::vector<double> srt(3 * nsources), trt(3 * ntargets);
        for (int64_t i = 0; i < nsources; ++i) {
            int32_t u = B.sperm[i];
            srt[i] = sx[u]; srt[nsources + i] = sy[u]; srt[2 * nsources + i] = sz[u];
        }
        const std::vector<int32_t> &tp = sat ? B.sperm : B.tperm;
        for (int64_t i = 0; i < ntargets; ++i) {
            int32_t u = tp[i];
            trt[i] = tx[u]; trt[ntargets + i] = ty[u]; trt[2 * ntargets + i] = tz[u];
        }
        std::vector<int32_t> user_source_ids(B.sperm.begin(), B.sperm.end());
        std::vector<int32_t> sorted_target_ids(ntargets);
        for (int64_t i = 0; i < ntargets; ++i) sorted_target_ids[tp[i]] = (int32_t)i;

        std::vector<double> centers(3 * nb);
        std::vector<int32_t> levels(nb), parent(nb), child(8 * nb, 0), coords(3 * nb);
        std::vector<int32_t> sstart(nb), scum(nb), snc(nb), tstart(nb), tcum(nb), tnc(nb);
        for (int64_t b = 0; b < nb; ++b) {
            const Box &x = B.boxes[b];
            double h = B.root_extent / (double)(1LL << x.level);
            for (int d = 0; d < 3; ++d) {
                centers[d * nb + b] = B.bbox_min[d] + (x.c[d] + 0.5) * h;
                coords[d * nb + b] = x.c[d];
            }
            levels[b] = x.level;
            parent[b] = x.parent < 0 ? 0 : x.parent;
            bool leaf = B.is_leaf((int32_t)b);
            for (int o = 0; o < 8; ++o) {
                int32_t c = B.children[8 * b + o];
                child[o * nb + b] = c < 0 ? 0 : c;
            }
            sstart[b] = (int32_t)x.s_lo; scum[b] = (int32_t)(x.s_hi - x.s_lo);
            snc[b] = leaf ? scum[b] : 0;
            tstart[b] = (int32_t)x.t_lo; tcum[b] = (int32_t)(x.t_hi - x.t_lo);
            tnc[b] = leaf ? tcum[b] : 0;
        }
        S->put_d("sources", std::move(srt));
        S->put_d("targets", std::move(trt));
        S->put_i("user_source_ids", std::move(user_source_ids));
        S->put_i("sorted_target_ids", std::move(sorted_target_ids));
        if (sat) {
            // tree-order target i is tree-order source i
            std::vector<int32_t> tts(nsources);
            std::iota(tts.begin(), tts.end(), 0);
            S->put_i("target_to_source", std::move(tts));
        }
        S->put_d("box_centers", std::move(centers));
        S->put_i("box_levels", std::move(levels));
        S->put_i("box_parent_ids", std::move(parent));
        S->put_i("box_child_ids", std::move(child));
        S->put_i("box_coords", std::move(coords));
        S->put_i("box_source_starts", std::move(sstart));
        S->put_i("box_source_counts_cumul", std::move(scum));
        S->put_i("box_source_counts_nonchild", std::move(snc));
        S->put_i("box_target_starts", std::move(tstart));
        S->put_i("box_target_counts_cumul", std::move(tcum));
        S->put_i("box_target_counts_nonchild", std::move(tnc));
        S->put_i("level_start_box_nrs", std::vector<int32_t>(B.level_start));
        S->put_d("bbox_min", std::vector<double>(B.bbox_min, B.bbox_min + 3));
        S->put_d("root_extent", std::vector<double>(1, B.root_extent));
        S->put_i("scalars", {(int32_t)nb, nl, (int32_t)nsources, (int32_t)ntargets, sat ? 1 : 0});

        // }}}

        // {{{ box sets

        std::vector<int32_t> source_boxes, target_boxes, source_parent_boxes, ttp_boxes;
        for (int64_t b = 0; b < nb; ++b) {
            bool leaf = B.is_leaf((int32_t)b);
            if (leaf && B.has_sources((int32_t)b)) source_boxes.push_back((int32_t)b);
            if (leaf && B.has_targets((int32_t)b)) target_boxes.push_back((int32_t)b);
            if (!leaf && B.has_sources((int32_t)b)) source_parent_boxes.push_back((int32_t)b);
            if (B.has_targets((int32_t)b)) ttp_boxes.push_back((int32_t)b);
        }
        auto level_starts = [&](const std::vector<int32_t> &bx) {
            std::vector<int32_t> ls(nl + 1, 0);
            size_t k = 0;
            for (int l = 0; l < nl; ++l) {
                ls[l] = (int32_t)k;
                while (k < bx.size() && B.boxes[bx[k]].level == l) ++k;
            }
            ls[nl] = (int32_t)k;
            return ls;
        };

        // }}}

        // {{{ colleagues (same-level adjacent boxes, self included)

        std::vector<std::vector<int32_t>> coll(nb);
        coll[0].push_back(0);
        for (int l = 1; l < nl; ++l) {
#pragma omp parallel for schedule(dynamic, 256)
            for (int32_t b = B.level_start[l]; b < B.level_start[l + 1]; ++b) {
                int32_t par = B.boxes[b].parent;
                for (int32_t pc : coll[par])
                    for (int o = 0; o < 8; ++o) {
                        int32_t c = B.children[8 * (size_t)pc + o];
                        if (c >= 0 && B.adjacent(c, b)) coll[b].push_back(c);
                    }
            }
        }

        // }}}

        // {{{ List 1 and List 3 (leaf target boxes)

        const int64_t ntb = (int64_t)target_boxes.size();
        std::vector<std::vector<int32_t>> l1(ntb), l3(ntb);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t it = 0; it < ntb; ++it) {
            int32_t t = target_boxes[it];
            std::vector<int32_t> stack;
            for (int32_t c : coll[t]) stack.push_back(c);
            while (!stack.empty()) {
                int32_t c = stack.back(); stack.pop_back();
                if (B.is_leaf(c)) {
                    if (B.has_sources(c)) l1[it].push_back(c);
                    continue;
                }
                for (int o = 0; o < 8; ++o) {
                    int32_t d = B.children[8 * (size_t)c + o];
                    if (d < 0) continue;
                    if (B.adjacent(d, t)) stack.push_back(d);
                    else if (B.has_sources(d)) l3[it].push_back(d);
                }
            }
            // coarser leaves adjacent to t: leaf colleagues of ancestors
            for (int32_t a = B.boxes[t].parent; a >= 0; a = B.boxes[a].parent) {
                for (int32_t c : coll[a])
                    if (c != a && B.is_leaf(c) && B.has_sources(c) && B.adjacent(c, t))
                        l1[it].push_back(c);
                if (a == 0) break;
            }
            std::sort(l1[it].begin(), l1[it].end());
            std::sort(l3[it].begin(), l3[it].end());
        }

        // }}}

        // {{{ List 2 and List 4 (target-or-target-parent boxes)

        const int64_t nttp = (int64_t)ttp_boxes.size();
        std::vector<std::vector<int32_t>> l2(nttp), l4(nttp), l2cls(nttp);
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t it = 0; it < nttp; ++it) {
            int32_t b = ttp_boxes[it];
            const Box &bx = B.boxes[b];
            if (bx.level < 1) continue;
            int32_t par = bx.parent;
            if (bx.level >= 2) {
                std::vector<std::pair<int32_t, int32_t>> ent;
                for (int32_t pc : coll[par])
                    for (int o = 0; o < 8; ++o) {
                        int32_t d = B.children[8 * (size_t)pc + o];
                        if (d < 0 || !B.has_sources(d)) continue;
                        const Box &dx = B.boxes[d];
                        int v[3] = {bx.c[0] - dx.c[0], bx.c[1] - dx.c[1], bx.c[2] - dx.c[2]};
                        if (std::abs(v[0]) <= 1 && std::abs(v[1]) <= 1 && std::abs(v[2]) <= 1) continue;
                        ent.push_back({d, class_of(v[0], v[1], v[2])});
                    }
                std::sort(ent.begin(), ent.end());
                for (auto &e : ent) { l2[it].push_back(e.first); l2cls[it].push_back(e.second); }
            }
            for (int32_t a = par; a >= 0; a = B.boxes[a].parent) {
                for (int32_t c : coll[a])
                    if (c != a && B.is_leaf(c) && B.has_sources(c) && B.adjacent(c, par) &&
                        !B.adjacent(c, b))
                        l4[it].push_back(c);
                if (a == 0) break;
            }
            std::sort(l4[it].begin(), l4[it].end());
        }

        // }}}

        // {{{ emit traversal

        std::vector<int32_t> st, fl;
        to_csr(l1, st, fl);
        S->put_i("neighbor_source_boxes_starts", st);
        S->put_i("neighbor_source_boxes_lists", fl);
        to_csr(l2, st, fl);
        S->put_i("from_sep_siblings_starts", st);
        S->put_i("from_sep_siblings_lists", fl);
        {
            std::vector<int32_t> cst, cfl;
            to_csr(l2cls, cst, cfl);
            // global class id = level * 316 + local class
            size_t k = 0;
            for (int64_t it = 0; it < nttp; ++it) {
                int lev = B.boxes[ttp_boxes[it]].level;
                for (size_t j = 0; j < l2cls[it].size(); ++j, ++k)
                    cfl[k] = (lev >= 2 ? (lev - 2) * NCLASSES : 0) + l2cls[it][j];
            }
            S->put_i("from_sep_siblings_translation_classes", std::move(cfl));
        }
        to_csr(l4, st, fl);
        S->put_i("from_sep_bigger_starts", st);
        S->put_i("from_sep_bigger_lists", fl);

        // List 3 split by source level
        std::vector<int32_t> l3_tb_level_starts(nl + 1, 0), l3_tb, l3_starts_all, l3_lists_all,
            l3_starts_level_offsets(nl + 1, 0), l3_lists_level_offsets(nl + 1, 0);
        for (int l = 0; l < nl; ++l) {
            l3_tb_level_starts[l] = (int32_t)l3_tb.size();
            l3_starts_level_offsets[l] = (int32_t)l3_starts_all.size();
            l3_lists_level_offsets[l] = (int32_t)l3_lists_all.size();
            int32_t run = 0;
            bool any = false;
            for (int64_t it = 0; it < ntb; ++it) {
                int cnt = 0;
                for (int32_t d : l3[it]) if (B.boxes[d].level == l) ++cnt;
                if (!cnt) continue;
                if (!any) { l3_starts_all.push_back(0); any = true; }
                l3_tb.push_back(target_boxes[it]);
                for (int32_t d : l3[it]) if (B.boxes[d].level == l) l3_lists_all.push_back(d);
                run += cnt;
                l3_starts_all.push_back(run);
            }
            if (!any) l3_starts_all.push_back(0);
        }
        l3_tb_level_starts[nl] = (int32_t)l3_tb.size();
        l3_starts_level_offsets[nl] = (int32_t)l3_starts_all.size();
        l3_lists_level_offsets[nl] = (int32_t)l3_lists_all.size();
        S->put_i("sep_smaller_target_boxes", std::move(l3_tb));
        S->put_i("sep_smaller_target_boxes_level_starts", std::move(l3_tb_level_starts));
        S->put_i("sep_smaller_starts", std::move(l3_starts_all));
        S->put_i("sep_smaller_starts_level_offsets", std::move(l3_starts_level_offsets));
        S->put_i("sep_smaller_lists", std::move(l3_lists_all));
        S->put_i("sep_smaller_lists_level_offsets", std::move(l3_lists_level_offsets));

        S->put_i("level_start_source_box_nrs", level_starts(source_boxes));
        S->put_i("level_start_target_box_nrs", level_starts(target_boxes));
        S->put_i("level_start_source_parent_box_nrs", level_starts(source_parent_boxes));
        S->put_i("level_start_target_or_target_parent_box_nrs", level_starts(ttp_boxes));
        S->put_i("source_boxes", std::move(source_boxes));
        S->put_i("target_boxes", std::move(target_boxes));
        S->put_i("source_parent_boxes", std::move(source_parent_boxes));
        S->put_i("target_or_target_parent_boxes", std::move(ttp_boxes));

        // translation classes: levels 0 and 1 have none
        std::vector<int32_t> cls_ls(nl + 1, 0);
        for (int l = 0; l < nl; ++l) cls_ls[l + 1] = cls_ls[l] + (l >= 2 ? NCLASSES : 0);
        std::vector<double> cvec(3 * (size_t)cls_ls[nl]);
        const int64_t ncl = cls_ls[nl];
        for (int l = 2; l < nl; ++l) {
            double h = B.root_extent / (double)(1LL << l);
            for (int a = -3; a <= 3; ++a)
                for (int b2 = -3; b2 <= 3; ++b2)
                    for (int c = -3; c <= 3; ++c) {
                        int k = class_of(a, b2, c);
                        if (k < 0) continue;
                        int64_t g = cls_ls[l] + k;
                        cvec[g] = a * h; cvec[ncl + g] = b2 * h; cvec[2 * ncl + g] = c * h;
                    }
        }
        S->put_i("from_sep_siblings_translation_classes_level_starts", std::move(cls_ls));
        S->put_d("from_sep_siblings_translation_class_to_distance_vector", std::move(cvec));

        // }}}

        *handle_out = S;
        return SUMPY_TREE_OK;
    } catch (const std::string &e) {
        g_last_error = e;
        return SUMPY_TREE_EINVAL;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return SUMPY_TREE_EINTERNAL;
    }
}

int sumpy_tree_array_info(void *handle, const char *name, int *kind, int64_t *length)
{
    auto *S = static_cast<TreeState *>(handle);
    if (!S || !name) { g_last_error = "null handle or name"; return SUMPY_TREE_EINVAL; }
    auto it = S->arrays.find(name);
    if (it == S->arrays.end()) { g_last_error = std::string("no tree array ") + name; return SUMPY_TREE_EINVAL; }
    *kind = it->second.kind;
    *length = it->second.kind == 0 ? (int64_t)it->second.i.size() : (int64_t)it->second.d.size();
    return SUMPY_TREE_OK;
}

int sumpy_tree_array_copy(void *handle, const char *name, void *dst, int64_t capacity_bytes)
{
    auto *S = static_cast<TreeState *>(handle);
    if (!S || !name || !dst) { g_last_error = "null argument"; return SUMPY_TREE_EINVAL; }
    auto it = S->arrays.find(name);
    if (it == S->arrays.end()) { g_last_error = std::string("no tree array ") + name; return SUMPY_TREE_EINVAL; }
    const Array &a = it->second;
    size_t bytes = a.kind == 0 ? a.i.size() * 4 : a.d.size() * 8;
    if ((int64_t)bytes > capacity_bytes) { g_last_error = "destination too small"; return SUMPY_TREE_EINVAL; }
    if (bytes) std::memcpy(dst, a.kind == 0 ? (const void *)a.i.data() : (const void *)a.d.data(), bytes);
    return SUMPY_TREE_OK;
}

void sumpy_tree_free(void *handle) { delete static_cast<TreeState *>(handle); }

int sumpy_pack_next_fit(int64_t n, const int32_t *sizes, int32_t capacity, int32_t max_count,
                        int32_t *item_first, int32_t *item_count, int64_t *nitems_out)
{
    if (n < 0 || capacity < 1 || max_count < 1 || !nitems_out || (n > 0 && !sizes) ||
        (n > 0 && (!item_first || !item_count))) {
        g_last_error = "pack_next_fit: bad arguments";
        return 1;
    }
    int64_t ni = 0, first = 0, cnt = 0, tot = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t r = sizes[i];
        if (cnt && (tot + r > capacity || cnt == max_count)) {
            item_first[ni] = (int32_t)first;
            item_count[ni] = (int32_t)cnt;
            ++ni;
            first = i;
            cnt = 0;
            tot = 0;
        }
        ++cnt;
        tot += r;
    }
    if (cnt) {
        item_first[ni] = (int32_t)first;
        item_count[ni] = (int32_t)cnt;
        ++ni;
    }
    *nitems_out = ni;
    return 0;
}

}  // extern "C"
