// Host-side planner: octrees and dual-tree interaction lists.
//
// The trees reproduce the reference's box indexing: Morton order of the
// points (zorder_less.hpp:212-248) realised with interleaved fixed-point keys,
// greedy closed-interval child ranges (octree.hpp:1106-1184) and per-level
// box ids in creation order.  The interaction lists follow the dual-tree walk
// of octree.hpp:255-349 in the same visiting order.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <new>
#include <utility>
#include <vector>

namespace ifgf
{

// Allocator whose resize leaves trivially constructible elements
// uninitialised: a vector sized here and then filled by several threads is
// not first zeroed (and paged in) on one thread.
template <typename T> struct UninitAlloc : std::allocator<T>
{
    using value_type = T;
    template <typename U> struct rebind
    {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <typename U> UninitAlloc(const UninitAlloc<U>&) noexcept {}
    template <typename U> void construct(U* p) { ::new ((void*)p) U; }
    template <typename U, typename... A> void construct(U* p, A&&... a)
    {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
};
template <typename T> using FillVector = std::vector<T, UninitAlloc<T>>;

struct TreeLevel
{
    std::vector<int64_t> first, last; // point range [first, last)
    std::vector<int32_t> parent;      // index in level-1 (-1 at the root)
    std::vector<uint8_t> leaf;
    std::vector<int32_t> child;       // 8 per box, index in level+1 or -1
    std::vector<double> bbmin, bbmax, center; // 3 per box
    double side = 0;                  // sideLength() of the first box (all equal)
    std::vector<double> sides;        // per box (identical up to rounding)
    size_t size() const { return first.size(); }
};

struct Tree
{
    int64_t n = 0;
    int64_t max_leaf = 100;
    std::vector<int64_t> perm;  // sorted position -> original index
    std::vector<double> pts;    // sorted points, AoS xyz
    std::vector<TreeLevel> levels;
    std::vector<int64_t> level_off; // global box id of the first box of a level

    int num_levels() const { return (int)levels.size(); }
    int64_t num_boxes_total() const { return level_off.empty() ? 0 : level_off.back(); }

    // Octree::build (octree.hpp:202-238) on the host
    void build(const double* p, int64_t n_pts, int64_t leaf_size);
    // The same tree built on the current GPU (gpu_tree.cu): Morton keys,
    // radix sort, and the children's point ranges of every level found by
    // one warp per box; the result equals build()'s bit for bit.
    void build_gpu(const double* p, int64_t n_pts, int64_t leaf_size);

    // Inflated bounding box of the points (octree.hpp:207-218), as build
    // computes it, from the plain coordinate minima and maxima.
    static void inflate_bbox(double* mn, double* mx);
    // Creates the levels from the sorted points (pts, perm set) and the root
    // box: the boxes of a level are split in id order, children in octant
    // order.  `split` fills, for every box b of the level with more than
    // max_leaf points, ends[8 b + j] = one past the last point of child j
    // (the greedy closed-interval scan of octree.hpp:1139-1170; a child is
    // empty when its end equals the previous child's).
    using SplitFn = std::function<void(const TreeLevel&, std::vector<int64_t>& ends)>;
    void make_levels(const double* mn, const double* mx, const SplitFn& split);
    // the child bounding box j of box b of level L (octree.hpp:1152-1163)
    static void child_box(const TreeLevel& L, size_t b, int j, double* cmn, double* cmx);
};

// Interaction lists in CSR form: the target boxes (global ids) of source
// box s (global id) are tgt[off[s] .. off[s + 1]), in discovery order.
struct PairLists
{
    std::vector<int64_t> off;
    std::vector<int32_t> tgt;
    int64_t count(int64_t s) const { return off[s + 1] - off[s]; }
    const int32_t* begin(int64_t s) const { return tgt.data() + off[s]; }
    const int32_t* end(int64_t s) const { return tgt.data() + off[s + 1]; }
    // CSR from pairs listed in discovery order (stable in each source box)
    void from_pairs(int64_t n_src_boxes, const std::vector<int32_t>& s,
                    const std::vector<int32_t>& t);
};

// Device copy of a source-major pair list: pair i's source and target
// global box ids, sources ascending and each source's targets in discovery
// order (the order of PairLists).  The buffers are freed with the last
// copy of the Plan.
struct DevicePairs
{
    std::shared_ptr<int32_t> src, tgt;
    int64_t n = 0;
};

struct Plan
{
    Tree src, tgt;
    PairLists far, near;
    // the same lists on the device: left there by the GPU walk, uploaded by
    // ensure_device_pairs after a host walk
    DevicePairs far_dev, near_dev;
    // target-leaf-centric lists for the evaluation kernel
    std::vector<int64_t> tleaf_gid;       // target leaves (global target box ids)
    std::vector<int64_t> tleaf_far_off;   // CSR offsets into tleaf_far_src
    FillVector<int32_t> tleaf_far_src;    // source global box ids
    std::vector<int64_t> tleaf_near_off;
    FillVector<int32_t> tleaf_near_src;   // source leaf global box ids
    // counters (octree.hpp:265-268)
    int64_t n_far_pairs = 0, n_near_pairs = 0, n_dropped = 0;
    int64_t far_target_evals = 0, near_point_pairs = 0;
    // Sharding of the matvec over ranks.  No source box above shard_level
    // has far targets, so the subtrees rooted at shard_level are
    // independent: each rank takes a contiguous (Morton-ordered) range of
    // them, balanced by modelled work, and computes their contribution to
    // every target.  box_rank: owning rank of every source box (boxes above
    // shard_level, whose only work is near-field leaves, belong to rank 0).
    int shard_level = 0;
    std::vector<int32_t> box_rank;

    void build_lists(const std::function<bool(double)>& cutoff);
    // The same lists (same order) from the dual-tree walk on the GPU, without
    // a cutoff predicate; false when the trees are too deep for its path keys
    // (the caller then walks on the host).
    bool build_lists_gpu();
    void assign_shards(int nranks);
    // Device copies of far and near (no-op where the GPU walk left them).
    void ensure_device_pairs();
    // tleaf_gid: the target leaves, by global box id
    void collect_target_leaves();
    // target-leaf lists of the sources owned by `rank` (all when rank < 0),
    // on the host (a plan-only init; the device tables are built from the
    // device pair lists by build_target_lists_gpu)
    void build_target_lists(int rank = -1);
    // Point-level work the target-leaf lists describe, for checking them
    // against the walk's lists: out[0] = sum over target leaves of (leaf
    // points x far-list length), out[1] = of (leaf points x points of each
    // far source box), out[2] = of (leaf points x points of each near source
    // leaf), and out[3] = sum over the far pairs (s, t) of the walk of
    // (points of s x points of t).  Without sharding out[0] equals
    // far_target_evals, out[1] equals out[3] and out[2] equals
    // near_point_pairs, since the leaves under a far pair's target box
    // partition its points; sharded, the ranks' out[0..2] add up to them.
    void target_list_work(int64_t out[4], uint64_t* checksum = nullptr) const;
    // the same from target-leaf lists given as arrays (the device tables
    // read back); checksum: a position-weighted sum of both lists, equal
    // for equal lists in equal order
    void target_list_work(const std::vector<long long>& far_off, const std::vector<int>& far_src,
                          const std::vector<long long>& near_off,
                          const std::vector<int>& near_src, int64_t out[4],
                          uint64_t* checksum) const;
    // Point range [first, last) of every target box, by global box id.
    void target_box_ranges(std::vector<int>& first, std::vector<int>& last) const;
    // Global id of the parent of every target box (-1 for the root).
    std::vector<int> target_parents() const;
};

// Reorders idx stably by key[idx[i]] -- the order std::stable_sort with a
// key comparison gives -- by a counting sort when every key is in
// [0, 2^26), else by std::stable_sort.
void stable_order_by_key(std::vector<int>& idx, const std::vector<int>& key);

// Morton key of a point normalised to the root box: 42 bits per dimension,
// interleaved z,y,x most significant first, split in two 63-bit halves.
void morton_key(const double* p, const double* center, const double* diam, uint64_t* hi,
                uint64_t* lo);

} // namespace ifgf
