// Host-side planner: octrees and dual-tree interaction lists.
#include "plan.hpp"

#include <algorithm>
#include <cmath>
#include <exception>
#include <numeric>
#include <system_error>
#include <thread>

#include "common.hpp"

namespace ifgf
{

// Spread the low 21 bits of v to every third bit position.
static inline uint64_t spread3(uint64_t v)
{
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// Order-preserving 42-bit code of a normalised coordinate p in (-0.5, 0.5):
// the top bit is the sign test of zorder_less.hpp:230 (negative first), the
// remaining 41 bits are |p| in fixed point, complemented for negative p so
// that larger magnitudes sort first, as `p[k] < q[k]` does for negatives.
static inline uint64_t coord_code(double p)
{
    const uint64_t top = 1ull << 41;
    const bool neg = p < 0.0;
    double a = std::fabs(p) * 4398046511104.0; // |p| * 2^42, exact scaling
    uint64_t u = a >= (double)(top - 1) ? top - 1 : (uint64_t)a;
    return neg ? (top - 1 - u) : (top | u);
}

void morton_key(const double* x, const double* c, const double* diam, uint64_t* hi,
                uint64_t* lo)
{
    // normalisation exactly as zorder_less.hpp:226-227
    uint64_t k[3];
    for (int d = 0; d < 3; d++)
        k[d] = coord_code((x[d] - c[d]) / diam[d]);
    // equal bit levels: z beats y beats x (ties keep the higher dimension,
    // zorder_less.hpp:229-240)
    *hi = (spread3(k[2] >> 21) << 2) | (spread3(k[1] >> 21) << 1) | spread3(k[0] >> 21);
    *lo = (spread3(k[2]) << 2) | (spread3(k[1]) << 1) | spread3(k[0]);
}

static bool box_contains(const double* mn, const double* mx, const double* p)
{
    for (int k = 0; k < 3; k++)
        if (!(mn[k] <= p[k]) || !(p[k] <= mx[k]))
            return false;
    return true;
}

void Tree::inflate_bbox(double* mn, double* mx)
{
    const double nmn = std::sqrt(mn[0] * mn[0] + mn[1] * mn[1] + mn[2] * mn[2]);
    const double nmx = std::sqrt(mx[0] * mx[0] + mx[1] * mx[1] + mx[2] * mx[2]);
    for (int d = 0; d < 3; d++)
    {
        mn[d] -= 1e-8 * nmn;
        mx[d] += 1e-8 * nmx;
    }
}

void Tree::child_box(const TreeLevel& L, size_t b, int j, double* cmn, double* cmx)
{
    for (int d = 0; d < 3; d++)
    {
        const double size = 0.5 * (L.bbmax[3 * b + d] - L.bbmin[3 * b + d]);
        cmn[d] = L.bbmin[3 * b + d] + size * (double)((j >> d) & 1);
        cmx[d] = cmn[d] + size;
    }
}

void Tree::build(const double* p, int64_t n_pts, int64_t leaf_size)
{
    n = n_pts;
    max_leaf = leaf_size;
    // bounding box, inflated as octree.hpp:207-218
    double mn[3], mx[3];
    for (int d = 0; d < 3; d++)
        mn[d] = mx[d] = p[d];
    for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++)
        {
            mn[d] = std::min(mn[d], p[3 * i + d]);
            mx[d] = std::max(mx[d], p[3 * i + d]);
        }
    inflate_bbox(mn, mx);
    double c[3], diam[3];
    for (int d = 0; d < 3; d++)
    {
        c[d] = (mx[d] + mn[d]) / 2.0;
        diam[d] = mx[d] - mn[d];
    }
    // Morton sort: keys, ties broken by the original index
    struct K
    {
        uint64_t hi, lo;
        int64_t idx;
    };
    std::vector<K> keys(n);
    for (int64_t i = 0; i < n; i++)
    {
        morton_key(p + 3 * i, c, diam, &keys[i].hi, &keys[i].lo);
        keys[i].idx = i;
    }
    std::sort(keys.begin(), keys.end(), [](const K& a, const K& b) {
        if (a.hi != b.hi)
            return a.hi < b.hi;
        if (a.lo != b.lo)
            return a.lo < b.lo;
        return a.idx < b.idx;
    });
    perm.resize(n);
    pts.resize(3 * n);
    for (int64_t i = 0; i < n; i++)
    {
        perm[i] = keys[i].idx;
        for (int d = 0; d < 3; d++)
            pts[3 * i + d] = p[3 * keys[i].idx + d];
    }
    keys.clear();
    keys.shrink_to_fit();
    // children's point ranges by the greedy scan over the sorted points
    make_levels(mn, mx, [&](const TreeLevel& L, std::vector<int64_t>& ends) {
        for (size_t b = 0; b < L.size(); b++)
        {
            if (L.last[b] - L.first[b] <= max_leaf)
                continue;
            int64_t pidx = L.first[b];
            for (int j = 0; j < 8; j++)
            {
                double cmn[3], cmx[3];
                child_box(L, b, j, cmn, cmx);
                while (pidx < L.last[b] && box_contains(cmn, cmx, &pts[3 * pidx]))
                    ++pidx;
                ends[8 * b + j] = pidx;
            }
        }
    });
}

void Tree::make_levels(const double* mn, const double* mx, const SplitFn& split)
{
    // Level-synchronous construction.  Visiting the boxes of a level in id
    // order and their children in octant order hands out the same per-level
    // ids as the depth-first construction of octree.hpp:1106-1184.
    levels.clear();
    auto push_box = [&](TreeLevel& L, int64_t f, int64_t l, int32_t par, const double* bmn,
                        const double* bmx) {
        L.first.push_back(f);
        L.last.push_back(l);
        L.parent.push_back(par);
        L.leaf.push_back(1);
        for (int j = 0; j < 8; j++)
            L.child.push_back(-1);
        double s = 0;
        for (int d = 0; d < 3; d++)
        {
            L.bbmin.push_back(bmn[d]);
            L.bbmax.push_back(bmx[d]);
            L.center.push_back((bmx[d] + bmn[d]) / 2.0);
            s = std::max(s, std::abs(bmx[d] - bmn[d]));
        }
        L.sides.push_back(s);
    };
    levels.emplace_back();
    if (n > 0)
        push_box(levels[0], 0, n, -1, mn, mx);
    std::vector<int64_t> ends;
    for (size_t l = 0; l < levels.size(); l++)
    {
        TreeLevel next;
        TreeLevel& L = levels[l];
        ends.assign(8 * L.size(), -1);
        split(L, ends);
        for (size_t b = 0; b < L.size(); b++)
        {
            const int64_t cnt = L.last[b] - L.first[b];
            if (cnt <= max_leaf)
                continue;
            int64_t pidx = L.first[b];
            for (int j = 0; j < 8; j++)
            {
                double cmn[3], cmx[3];
                child_box(L, b, j, cmn, cmx);
                const int64_t end = ends[8 * b + j];
                if (end > pidx)
                {
                    L.child[8 * b + j] = (int32_t)next.size();
                    L.leaf[b] = 0;
                    push_box(next, pidx, end, (int32_t)b, cmn, cmx);
                }
                pidx = end;
            }
        }
        if (next.size() == 0)
            break;
        levels.push_back(std::move(next));
    }
    level_off.assign(levels.size() + 1, 0);
    for (size_t l = 0; l < levels.size(); l++)
    {
        levels[l].side = levels[l].size() ? levels[l].sides[0] : 0;
        level_off[l + 1] = level_off[l] + (int64_t)levels[l].size();
    }
}

namespace
{
struct Walker
{
    Plan& P;
    const std::function<bool(double)>& cutoff;
    const double eta = std::sqrt(3.0);
    // (source, target) global box ids of the far and near pairs, in discovery order
    std::vector<int32_t> fs, ft, ns, nt;

    // Octree::buildInteractionList (octree.hpp:272-349)
    void walk(int sl, int32_t s, int tl, int32_t t)
    {
        if (s < 0 || t < 0)
            return;
        const TreeLevel& SL = P.src.levels[sl];
        const TreeLevel& TL = P.tgt.levels[tl];
        if (SL.first[s] == SL.last[s] || TL.first[t] == TL.last[t])
            return;
        // admissibility (octree.hpp:189-198): exterior distance of the
        // target box to the source centre >= sqrt(3) * source side length
        double d2 = 0;
        for (int k = 0; k < 3; k++)
        {
            const double p = SL.center[3 * s + k];
            const double lo = TL.bbmin[3 * t + k], hi = TL.bbmax[3 * t + k];
            if (lo > p)
            {
                const double a = lo - p;
                d2 += a * a;
            }
            else if (p > hi)
            {
                const double a = p - hi;
                d2 += a * a;
            }
        }
        const double dist = std::sqrt(d2);
        const int64_t sg = P.src.level_off[sl] + s, tg = P.tgt.level_off[tl] + t;
        if (dist >= eta * SL.sides[s])
        {
            if (cutoff && cutoff(dist))
            {
                P.n_dropped++;
                return;
            }
            fs.push_back((int32_t)sg);
            ft.push_back((int32_t)tg);
            P.n_far_pairs++;
            P.far_target_evals += TL.last[t] - TL.first[t];
            return;
        }
        const bool sleaf = SL.leaf[s], tleaf = TL.leaf[t];
        if (sleaf && tleaf)
        {
            ns.push_back((int32_t)sg);
            nt.push_back((int32_t)tg);
            P.n_near_pairs++;
            P.near_point_pairs += (SL.last[s] - SL.first[s]) * (TL.last[t] - TL.first[t]);
            return;
        }
        if (sleaf && !tleaf)
        {
            for (int j = 0; j < 8; j++)
                walk(sl, s, tl + 1, TL.child[8 * t + j]);
            return;
        }
        if (tleaf && !sleaf)
        {
            for (int j = 0; j < 8; j++)
                walk(sl + 1, SL.child[8 * s + j], tl, t);
            return;
        }
        if (SL.sides[s] > TL.sides[t])
            for (int j = 0; j < 8; j++)
                walk(sl + 1, SL.child[8 * s + j], tl, t);
        else
            for (int j = 0; j < 8; j++)
                walk(sl, s, tl + 1, TL.child[8 * t + j]);
    }
};
} // namespace

void PairLists::from_pairs(int64_t n_src_boxes, const std::vector<int32_t>& s,
                           const std::vector<int32_t>& t)
{
    off.assign(n_src_boxes + 1, 0);
    for (int32_t x : s)
        off[x + 1]++;
    for (int64_t i = 0; i < n_src_boxes; i++)
        off[i + 1] += off[i];
    tgt.resize(t.size());
    std::vector<int64_t> at(off.begin(), off.end() - 1);
    for (size_t i = 0; i < s.size(); i++)
        tgt[at[s[i]]++] = t[i];
}

void Plan::build_lists(const std::function<bool(double)>& cutoff)
{
    const int64_t nb = src.num_boxes_total();
    n_far_pairs = n_near_pairs = n_dropped = far_target_evals = near_point_pairs = 0;
    far_dev = near_dev = DevicePairs{}; // device copies of earlier lists
    Walker w{*this, cutoff};
    if (src.n > 0 && tgt.n > 0)
        w.walk(0, 0, 0, 0);
    far.from_pairs(nb, w.fs, w.ft);
    near.from_pairs(nb, w.ns, w.nt);
}

void Plan::assign_shards(int nranks)
{
    const int L = src.num_levels();
    const int64_t nsb = src.num_boxes_total();
    // first level with a far pair (the subtree roots)
    shard_level = L - 1;
    for (int l = 0; l < L; l++)
    {
        bool any = false;
        for (size_t b = 0; b < src.levels[l].size() && !any; b++)
            any = far.count(src.level_off[l] + (int64_t)b) > 0;
        if (any)
        {
            shard_level = l;
            break;
        }
    }
    box_rank.assign(nsb, 0);
    if (nranks <= 1)
        return;
    // modelled work of every box: near point pairs + far target evaluations
    // weighted by the cost of one evaluation relative to one kernel pair
    auto tsize = [&](int64_t tg) {
        int l = (int)(std::upper_bound(tgt.level_off.begin(), tgt.level_off.end(), tg) -
                      tgt.level_off.begin()) - 1;
        const int64_t b = tg - tgt.level_off[l];
        return (double)(tgt.levels[l].last[b] - tgt.levels[l].first[b]);
    };
    std::vector<double> work(nsb, 0.0);
    for (int l = L - 1; l >= 0; l--)
        for (size_t b = 0; b < src.levels[l].size(); b++)
        {
            const int64_t g = src.level_off[l] + (int64_t)b;
            const double ns = (double)(src.levels[l].last[b] - src.levels[l].first[b]);
            for (const int32_t* t = near.begin(g); t != near.end(g); t++)
                work[g] += ns * tsize(*t);
            for (const int32_t* t = far.begin(g); t != far.end(g); t++)
                work[g] += 20.0 * tsize(*t);
            if (l > 0)
                work[src.level_off[l - 1] + src.levels[l].parent[b]] += work[g];
        }
    const TreeLevel& S = src.levels[shard_level];
    const int64_t nr = (int64_t)S.size();
    double total = 0;
    for (int64_t b = 0; b < nr; b++)
        total += work[src.level_off[shard_level] + b];
    // contiguous ranges: rank r ends where the running work passes
    // (r + 1) / nranks of the total
    std::vector<int32_t> root_rank(nr, 0);
    double run = 0;
    int r = 0;
    for (int64_t b = 0; b < nr; b++)
    {
        const double wb = work[src.level_off[shard_level] + b];
        while (r < nranks - 1 && run + 0.5 * wb > total * (double)(r + 1) / nranks)
            r++;
        root_rank[b] = r;
        run += wb;
    }
    for (int64_t b = 0; b < nr; b++)
        box_rank[src.level_off[shard_level] + b] = root_rank[b];
    for (int l = shard_level + 1; l < L; l++)
        for (size_t b = 0; b < src.levels[l].size(); b++)
            box_rank[src.level_off[l] + (int64_t)b] =
                box_rank[src.level_off[l - 1] + src.levels[l].parent[b]];
}

namespace
{
// Joins the given threads when it goes out of scope, so that no joinable
// std::thread is destroyed (which would end the process) when an exception
// leaves the scope that started them.
struct JoinAll
{
    std::thread* one;
    int n_one;
    std::vector<std::thread>* many = nullptr;
    ~JoinAll()
    {
        for (int i = 0; i < n_one; i++)
            if (one[i].joinable())
                one[i].join();
        if (many)
            for (auto& t : *many)
                if (t.joinable())
                    t.join();
    }
};
} // namespace

void Plan::build_target_lists(int rank)
{
    const int64_t ntb = tgt.num_boxes_total();
    const int64_t nsb = src.num_boxes_total();
    // transpose to per-target CSR (sources ascending), counting sort
    auto transpose = [&](const PairLists& in, std::vector<int64_t>& off,
                         std::vector<int32_t>& srcs) {
        off.assign(ntb + 1, 0);
        for (int64_t s = 0; s < nsb; s++)
            if (rank < 0 || box_rank[s] == rank)
                for (const int32_t* t = in.begin(s); t != in.end(s); t++)
                    off[*t + 1]++;
        for (int64_t i = 0; i < ntb; i++)
            off[i + 1] += off[i];
        srcs.resize(off[ntb]);
        std::vector<int64_t> at(off.begin(), off.end() - 1);
        for (int64_t s = 0; s < nsb; s++)
            if (rank < 0 || box_rank[s] == rank)
                for (const int32_t* t = in.begin(s); t != in.end(s); t++)
                    srcs[at[*t]++] = (int32_t)s;
    };
    std::vector<int64_t> fin_off, nin_off;
    std::vector<int32_t> fin, nin;
    // the two transposes are independent: for large lists the near one runs
    // on a second thread when one can be had.  The thread is joined on every
    // path out of this block (an exception from the far transpose included),
    // and an exception inside it is carried back to this thread.
    {
        std::exception_ptr near_err;
        std::thread near_thread;
        JoinAll guard{&near_thread, 1};
        if (near.tgt.size() + far.tgt.size() > ((size_t)1 << 18))
        {
            try
            {
                near_thread = std::thread([&] {
                    try
                    {
                        transpose(near, nin_off, nin);
                    }
                    catch (...)
                    {
                        near_err = std::current_exception();
                    }
                });
            }
            catch (const std::system_error&)
            {
            }
        }
        if (!near_thread.joinable())
            transpose(near, nin_off, nin);
        transpose(far, fin_off, fin);
        if (near_thread.joinable())
            near_thread.join();
        if (near_err)
            std::rethrow_exception(near_err);
    }
    // A target leaf's far list is the concatenation of its own far sources
    // and those of every ancestor, leaf first.  Count them per box, parents
    // before children (cum = own + parent's cum), so the CSR is sized exactly
    // before it is filled.
    const int L = tgt.num_levels();
    std::vector<int64_t> cum((size_t)ntb, 0);
    collect_target_leaves();
    for (int l = 0; l < L; l++)
    {
        const TreeLevel& TL = tgt.levels[l];
        const int64_t o = tgt.level_off[l];
        for (size_t b = 0; b < TL.size(); b++)
        {
            const int64_t g = o + (int64_t)b;
            cum[g] = fin_off[g + 1] - fin_off[g] +
                     (l > 0 ? cum[tgt.level_off[l - 1] + TL.parent[b]] : 0);
        }
    }
    const int64_t nl = (int64_t)tleaf_gid.size();
    tleaf_far_off.assign((size_t)nl + 1, 0);
    tleaf_near_off.assign((size_t)nl + 1, 0);
    for (int64_t i = 0; i < nl; i++)
    {
        const int64_t g = tleaf_gid[i];
        tleaf_far_off[i + 1] = tleaf_far_off[i] + cum[g];
        tleaf_near_off[i + 1] = tleaf_near_off[i] + (nin_off[g + 1] - nin_off[g]);
    }
    tleaf_far_src.resize((size_t)tleaf_far_off[nl]);
    tleaf_near_src.resize((size_t)tleaf_near_off[nl]);
    // global target box id -> (level, index in level)
    std::vector<int32_t> box_level((size_t)ntb);
    for (int l = 0; l < L; l++)
        std::fill(box_level.begin() + tgt.level_off[l], box_level.begin() + tgt.level_off[l + 1], l);
    // Fill leaves [lo, hi): every leaf writes its own slice, so threads
    // given disjoint leaf ranges need no synchronisation.
    auto fill = [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; i++)
        {
            const int64_t g = tleaf_gid[i];
            int32_t* out = tleaf_far_src.data() + tleaf_far_off[i];
            int al = box_level[g];
            int32_t ab = (int32_t)(g - tgt.level_off[al]);
            while (al >= 0)
            {
                const int64_t ag = tgt.level_off[al] + ab;
                out = std::copy(fin.begin() + fin_off[ag], fin.begin() + fin_off[ag + 1], out);
                ab = tgt.levels[al].parent[ab];
                al--;
            }
            std::copy(nin.begin() + nin_off[g], nin.begin() + nin_off[g + 1],
                      tleaf_near_src.begin() + tleaf_near_off[i]);
        }
    };
    // Leaf ranges of about equal far-entry counts; small plans stay on the
    // calling thread.
    const int64_t total = tleaf_far_off[nl] + tleaf_near_off[nl];
    const int nt = (int)std::min<int64_t>(
        std::max(1u, std::min(16u, std::thread::hardware_concurrency())), 1 + total / (1 << 20));
    if (nt <= 1)
    {
        fill(0, nl);
        return;
    }
    std::vector<int64_t> cut((size_t)nt + 1, nl);
    cut[0] = 0;
    for (int t = 1; t < nt; t++)
    {
        const int64_t want = tleaf_far_off[nl] * t / nt;
        cut[t] = std::lower_bound(tleaf_far_off.begin(), tleaf_far_off.end(), want) -
                 tleaf_far_off.begin();
        cut[t] = std::max(cut[t - 1], std::min(cut[t], nl));
    }
    // fill() only copies into sized arrays, so the workers cannot throw; the
    // joiner joins every started worker on every path out of this function
    std::vector<std::thread> pool;
    pool.reserve((size_t)nt);
    JoinAll guard{nullptr, 0, &pool};
    for (int t = 1; t < nt; t++)
    {
        try
        {
            pool.emplace_back(fill, cut[t], cut[t + 1]);
        }
        catch (const std::system_error&) // no thread to be had: fill here
        {
            fill(cut[t], cut[t + 1]);
        }
    }
    fill(cut[0], cut[1]);
}

void Plan::collect_target_leaves()
{
    tleaf_gid.clear();
    for (int l = 0; l < tgt.num_levels(); l++)
        for (size_t b = 0; b < tgt.levels[l].size(); b++)
            if (tgt.levels[l].leaf[b])
                tleaf_gid.push_back(tgt.level_off[l] + (int64_t)b);
}

std::vector<int> Plan::target_parents() const
{
    std::vector<int> par((size_t)tgt.num_boxes_total(), -1);
    for (int l = 1; l < tgt.num_levels(); l++)
        for (size_t b = 0; b < tgt.levels[l].size(); b++)
            par[tgt.level_off[l] + (int64_t)b] =
                (int)(tgt.level_off[l - 1] + tgt.levels[l].parent[b]);
    return par;
}

void Plan::target_list_work(const std::vector<long long>& far_off, const std::vector<int>& far_src,
                            const std::vector<long long>& near_off,
                            const std::vector<int>& near_src, int64_t out[4],
                            uint64_t* checksum) const
{
    auto points = [](const Tree& T) {
        std::vector<int64_t> n((size_t)T.num_boxes_total());
        for (int l = 0; l < T.num_levels(); l++)
            for (size_t b = 0; b < T.levels[l].size(); b++)
                n[T.level_off[l] + (int64_t)b] = T.levels[l].last[b] - T.levels[l].first[b];
        return n;
    };
    const std::vector<int64_t> ps = points(src), pt = points(tgt);
    int64_t fe = 0, fp = 0, np = 0;
    uint64_t h = 0;
    for (size_t i = 0; i < tleaf_gid.size(); i++)
    {
        const int64_t nt = pt[tleaf_gid[i]];
        fe += nt * (far_off[i + 1] - far_off[i]);
        for (long long j = far_off[i]; j < far_off[i + 1]; j++)
        {
            fp += nt * ps[far_src[j]];
            h = h * 1000003ull + (uint64_t)(far_src[j] + 1) * (uint64_t)(j + 1);
        }
        for (long long j = near_off[i]; j < near_off[i + 1]; j++)
        {
            np += nt * ps[near_src[j]];
            h = h * 998244353ull + (uint64_t)(near_src[j] + 1) * (uint64_t)(j + 7);
        }
        h ^= (uint64_t)far_off[i + 1] * 31ull + (uint64_t)near_off[i + 1];
    }
    int64_t wp = 0;
    const int64_t nsb = src.num_boxes_total();
    for (int64_t s = 0; s < nsb && !far.off.empty(); s++)
        for (const int32_t* t = far.begin(s); t != far.end(s); t++)
            wp += ps[s] * pt[*t];
    out[0] = fe;
    out[1] = fp;
    out[2] = np;
    out[3] = wp;
    if (checksum)
        *checksum = h;
}

void Plan::target_list_work(int64_t out[4], uint64_t* checksum) const
{
    const std::vector<long long> fo(tleaf_far_off.begin(), tleaf_far_off.end()),
        no(tleaf_near_off.begin(), tleaf_near_off.end());
    const std::vector<int> fs(tleaf_far_src.begin(), tleaf_far_src.end()),
        ns(tleaf_near_src.begin(), tleaf_near_src.end());
    target_list_work(fo, fs, no, ns, out, checksum);
}

void Plan::target_box_ranges(std::vector<int>& first, std::vector<int>& last) const
{
    const int64_t ntb = tgt.num_boxes_total();
    first.resize((size_t)ntb);
    last.resize((size_t)ntb);
    for (int l = 0; l < tgt.num_levels(); l++)
        for (size_t b = 0; b < tgt.levels[l].size(); b++)
        {
            first[tgt.level_off[l] + (int64_t)b] = (int)tgt.levels[l].first[b];
            last[tgt.level_off[l] + (int64_t)b] = (int)tgt.levels[l].last[b];
        }
}

void stable_order_by_key(std::vector<int>& idx, const std::vector<int>& key)
{
    int kmax = -1;
    bool counting = true;
    for (int i : idx)
    {
        const int k = key[i];
        if (k < 0 || k >= (1 << 26))
        {
            counting = false;
            break;
        }
        kmax = std::max(kmax, k);
    }
    // a counting array much longer than the list would cost more than it
    // saves: keys spread that widely take the comparison sort
    if (counting && (int64_t)kmax > 4 * (int64_t)idx.size() + 4096)
        counting = false;
    if (!counting)
    {
        std::stable_sort(idx.begin(), idx.end(),
                         [&](int a, int b) { return key[a] < key[b]; });
        return;
    }
    std::vector<int64_t> at((size_t)kmax + 2, 0);
    for (int i : idx)
        at[key[i] + 1]++;
    for (size_t k = 1; k < at.size(); k++)
        at[k] += at[k - 1];
    std::vector<int> out(idx.size());
    for (int i : idx)
        out[at[key[i]]++] = i;
    idx.swap(out);
}

} // namespace ifgf
