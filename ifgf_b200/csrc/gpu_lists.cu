// Interaction lists on the GPU (Plan::build_lists_gpu): the dual-tree walk of
// Octree::buildInteractionList (octree.hpp:272-349) as a level-synchronous
// expansion of (source box, target box) pairs.
//   * One kernel per step classifies every pair of the frontier: dropped
//     (an empty box), far (exterior distance of the target box to the source
//     centre >= sqrt(3) x the source side, octree.hpp:189-198), near (two
//     leaves), or split (the leaf-less or larger box, ties splitting the
//     target) into its existing children, which form the next frontier.
//     The distance uses explicitly rounded FP64 operations in the host
//     walker's order, so every decision equals the host's.
//   * Each pair carries its path from the root pair: the child index chosen
//     at every split, 3 bits per step, most significant first (two 63-bit
//     words, 42 steps).  The recursive walk discovers pairs in lexicographic
//     order of these paths, so sorting the far and near pairs by (source box,
//     path) -- three stable radix sorts -- gives every source box its list in
//     the host walker's order.
//   * Output slots come from atomic counters; a step whose outputs overflow
//     the buffers is run again after they grow.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "common.hpp"
#include "plan.hpp"

namespace ifgf
{
namespace
{

#define LIST_CUDA(x)                                                                          \
    do                                                                                         \
    {                                                                                          \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            throw Error(2, std::string("interaction lists: ") + #x + ": " +                    \
                               cudaGetErrorString(e_));                                        \
    } while (0)

template <typename T> struct LBuf
{
    T* p = nullptr;
    size_t n = 0;
    LBuf() = default;
    LBuf(const LBuf&) = delete;
    LBuf& operator=(const LBuf&) = delete;
    ~LBuf()
    {
        if (p)
            cudaFree(p);
    }
    void alloc(size_t count)
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        n = std::max<size_t>(count, 1);
        LIST_CUDA(cudaMalloc((void**)&p, n * sizeof(T)));
    }
    // larger buffer keeping the first `keep` entries
    void grow(size_t count, size_t keep)
    {
        if (count <= n)
            return;
        T* q = nullptr;
        LIST_CUDA(cudaMalloc((void**)&q, count * sizeof(T)));
        if (p && keep)
            LIST_CUDA(cudaMemcpy(q, p, std::min(keep, n) * sizeof(T), cudaMemcpyDeviceToDevice));
        if (p)
            cudaFree(p);
        p = q;
        n = count;
    }
    // hands the allocation over to the caller
    T* release()
    {
        T* q = p;
        p = nullptr;
        n = 0;
        return q;
    }
    void swap(LBuf& o)
    {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
    void upload(const std::vector<T>& v)
    {
        alloc(v.size());
        if (!v.empty())
            LIST_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
};

// boxes of both trees by global id
struct WalkTrees
{
    const double* sc;     // source centres, xyz
    const double* sside;  // source side lengths
    const int64_t* sfirst;
    const int64_t* slast;
    const uint8_t* sleaf;
    const int32_t* schild; // 8 per box: global id or -1
    const double* tmin;    // target bounding boxes, xyz
    const double* tmax;
    const double* tside;
    const int64_t* tfirst;
    const int64_t* tlast;
    const uint8_t* tleaf;
    const int32_t* tchild;
    double eta;
};

// a list of pairs with their paths
struct PairBuf
{
    int32_t* s;
    int32_t* t;
    uint64_t* k0;
    uint64_t* k1;
};

// counters: next frontier, far pairs, near pairs, far target evaluations,
// near point pairs
enum
{
    C_NEXT = 0,
    C_FAR,
    C_NEAR,
    C_FAR_EVALS,
    C_NEAR_PAIRS,
    C_COUNT
};

__global__ void __launch_bounds__(256) walk_step_kernel(WalkTrees T, PairBuf in, long long n_in,
                                                        int step, PairBuf next,
                                                        long long cap_next, PairBuf far,
                                                        long long cap_far, PairBuf near,
                                                        long long cap_near,
                                                        unsigned long long* ctr)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n_in)
        return;
    const int32_t s = in.s[i], t = in.t[i];
    const uint64_t k0 = in.k0[i], k1 = in.k1[i];
    const long long sn = T.slast[s] - T.sfirst[s], tn = T.tlast[t] - T.tfirst[t];
    if (sn == 0 || tn == 0)
        return;
    // admissibility, in the host walker's operation order without contraction
    double d2 = 0;
    for (int k = 0; k < 3; k++)
    {
        const double p = T.sc[3 * s + k];
        const double lo = T.tmin[3 * t + k], hi = T.tmax[3 * t + k];
        if (lo > p)
        {
            const double a = __dsub_rn(lo, p);
            d2 = __dadd_rn(d2, __dmul_rn(a, a));
        }
        else if (p > hi)
        {
            const double a = __dsub_rn(p, hi);
            d2 = __dadd_rn(d2, __dmul_rn(a, a));
        }
    }
    const double dist = __dsqrt_rn(d2);
    if (dist >= __dmul_rn(T.eta, T.sside[s]))
    {
        const unsigned long long slot = atomicAdd(&ctr[C_FAR], 1ull);
        atomicAdd(&ctr[C_FAR_EVALS], (unsigned long long)tn);
        if (slot < (unsigned long long)cap_far)
        {
            far.s[slot] = s;
            far.t[slot] = t;
            far.k0[slot] = k0;
            far.k1[slot] = k1;
        }
        return;
    }
    const bool sl = T.sleaf[s], tl = T.tleaf[t];
    if (sl && tl)
    {
        const unsigned long long slot = atomicAdd(&ctr[C_NEAR], 1ull);
        atomicAdd(&ctr[C_NEAR_PAIRS], (unsigned long long)(sn * tn));
        if (slot < (unsigned long long)cap_near)
        {
            near.s[slot] = s;
            near.t[slot] = t;
            near.k0[slot] = k0;
            near.k1[slot] = k1;
        }
        return;
    }
    const bool split_s = !sl && (tl || T.sside[s] > T.tside[t]);
    const int32_t* ch = split_s ? T.schild + 8 * (size_t)s : T.tchild + 8 * (size_t)t;
    int nvalid = 0;
    for (int j = 0; j < 8; j++)
        nvalid += ch[j] >= 0;
    if (nvalid == 0)
        return;
    unsigned long long pos = atomicAdd(&ctr[C_NEXT], (unsigned long long)nvalid);
    const int shift = 60 - 3 * (step % 21);
    for (int j = 0; j < 8; j++)
    {
        const int32_t c = ch[j];
        if (c < 0)
            continue;
        if (pos < (unsigned long long)cap_next)
        {
            next.s[pos] = split_s ? c : s;
            next.t[pos] = split_s ? t : c;
            const uint64_t d = (uint64_t)j << shift;
            next.k0[pos] = step < 21 ? (k0 | d) : k0;
            next.k1[pos] = step >= 21 && step < 42 ? (k1 | d) : k1;
        }
        pos++;
    }
}

template <typename T>
__global__ void gather_kernel(const T* __restrict__ in, const int* __restrict__ idx, T* out,
                              long long n)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = in[idx[i]];
}

__global__ void iota_kernel(int* v, long long n)
{
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n)
        v[i] = (int)i;
}

unsigned grid_for(long long n) { return (unsigned)((n + 255) / 256); }

template <typename T> std::shared_ptr<T> device_owned(T* p)
{
    return std::shared_ptr<T>(p, [](T* q) { cudaFree(q); });
}

// (source, target) pairs ordered by (source, k0, k1), as CSR on the host and
// as (source, target) arrays left on the device
void sort_to_csr(const PairBuf& pb, long long n, int64_t n_src_boxes, PairLists& out,
                 DevicePairs& dev)
{
    out.off.assign(n_src_boxes + 1, 0);
    out.tgt.clear();
    dev = DevicePairs{};
    if (n == 0)
        return;
    LBuf<int> ia, ib;
    LBuf<uint64_t> ka, kb;
    LBuf<int32_t> sa, sb;
    ia.alloc(n);
    ib.alloc(n);
    ka.alloc(n);
    kb.alloc(n);
    sa.alloc(n);
    sb.alloc(n);
    iota_kernel<<<grid_for(n), 256>>>(ia.p, n);
    LIST_CUDA(cudaGetLastError());
    size_t tb = 0, tb2 = 0;
    LIST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, ka.p, kb.p, ia.p, ib.p, (int)n));
    LIST_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb2, sa.p, sb.p, ia.p, ib.p, (int)n));
    LBuf<unsigned char> tmp;
    tmp.alloc(std::max(tb, tb2));
    // stable passes: k1, then k0, then the source box
    LIST_CUDA(cudaMemcpy(ka.p, pb.k1, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice));
    LIST_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, ka.p, kb.p, ia.p, ib.p, (int)n));
    gather_kernel<<<grid_for(n), 256>>>(pb.k0, ib.p, ka.p, n);
    LIST_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, ka.p, kb.p, ib.p, ia.p, (int)n));
    gather_kernel<<<grid_for(n), 256>>>(pb.s, ia.p, sa.p, n);
    LIST_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb2, sa.p, sb.p, ia.p, ib.p, (int)n));
    gather_kernel<<<grid_for(n), 256>>>(pb.t, ib.p, sa.p, n);
    LIST_CUDA(cudaGetLastError());
    std::vector<int32_t> s_sorted(n);
    out.tgt.resize(n);
    LIST_CUDA(cudaMemcpy(s_sorted.data(), sb.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    LIST_CUDA(cudaMemcpy(out.tgt.data(), sa.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    for (long long i = 0; i < n; i++)
        out.off[s_sorted[i] + 1]++;
    for (int64_t b = 0; b < n_src_boxes; b++)
        out.off[b + 1] += out.off[b];
    dev.src = device_owned(sb.release());
    dev.tgt = device_owned(sa.release());
    dev.n = n;
}

} // namespace

bool Plan::build_lists_gpu()
{
    const int Ls = src.num_levels(), Lt = tgt.num_levels();
    if (Ls + Lt - 2 > 42)
        return false; // paths longer than two key words: the host walk
    n_far_pairs = n_near_pairs = n_dropped = far_target_evals = near_point_pairs = 0;
    const int64_t nsb = src.num_boxes_total(), ntb = tgt.num_boxes_total();
    if (src.n == 0 || tgt.n == 0)
    {
        far.from_pairs(nsb, {}, {});
        near.from_pairs(nsb, {}, {});
        return true;
    }
    // both trees by global box id
    std::vector<double> sc(3 * nsb), sside(nsb), tmin(3 * ntb), tmax(3 * ntb), tside(ntb);
    std::vector<int64_t> sfirst(nsb), slast(nsb), tfirst(ntb), tlast(ntb);
    std::vector<uint8_t> sleaf(nsb), tleaf(ntb);
    std::vector<int32_t> schild(8 * nsb), tchild(8 * ntb);
    auto flatten = [](const Tree& tr, double* c3, double* mn3, double* mx3, double* side,
                      int64_t* first, int64_t* last, uint8_t* leaf, int32_t* child) {
        const int L = tr.num_levels();
        for (int l = 0; l < L; l++)
        {
            const TreeLevel& TL = tr.levels[l];
            const int64_t off = tr.level_off[l];
            const int64_t coff = l + 1 < L ? tr.level_off[l + 1] : 0;
            for (size_t b = 0; b < TL.size(); b++)
            {
                const int64_t g = off + (int64_t)b;
                for (int d = 0; d < 3; d++)
                {
                    if (c3)
                        c3[3 * g + d] = TL.center[3 * b + d];
                    if (mn3)
                    {
                        mn3[3 * g + d] = TL.bbmin[3 * b + d];
                        mx3[3 * g + d] = TL.bbmax[3 * b + d];
                    }
                }
                side[g] = TL.sides[b];
                first[g] = TL.first[b];
                last[g] = TL.last[b];
                leaf[g] = TL.leaf[b];
                for (int j = 0; j < 8; j++)
                {
                    const int32_t c = TL.child[8 * b + j];
                    child[8 * g + j] = c < 0 ? -1 : (int32_t)(coff + c);
                }
            }
        }
    };
    flatten(src, sc.data(), nullptr, nullptr, sside.data(), sfirst.data(), slast.data(),
            sleaf.data(), schild.data());
    flatten(tgt, nullptr, tmin.data(), tmax.data(), tside.data(), tfirst.data(), tlast.data(),
            tleaf.data(), tchild.data());
    LBuf<double> d_sc, d_sside, d_tmin, d_tmax, d_tside;
    LBuf<int64_t> d_sfirst, d_slast, d_tfirst, d_tlast;
    LBuf<uint8_t> d_sleaf, d_tleaf;
    LBuf<int32_t> d_schild, d_tchild;
    d_sc.upload(sc);
    d_sside.upload(sside);
    d_tmin.upload(tmin);
    d_tmax.upload(tmax);
    d_tside.upload(tside);
    d_sfirst.upload(sfirst);
    d_slast.upload(slast);
    d_tfirst.upload(tfirst);
    d_tlast.upload(tlast);
    d_sleaf.upload(sleaf);
    d_tleaf.upload(tleaf);
    d_schild.upload(schild);
    d_tchild.upload(tchild);
    const WalkTrees T{d_sc.p,     d_sside.p,  d_sfirst.p, d_slast.p, d_sleaf.p,
                      d_schild.p, d_tmin.p,   d_tmax.p,   d_tside.p, d_tfirst.p,
                      d_tlast.p,  d_tleaf.p,  d_tchild.p, std::sqrt(3.0)};

    struct Lists
    {
        LBuf<int32_t> s, t;
        LBuf<uint64_t> k0, k1;
        void alloc(size_t n)
        {
            s.alloc(n);
            t.alloc(n);
            k0.alloc(n);
            k1.alloc(n);
        }
        void grow(size_t n, size_t keep)
        {
            s.grow(n, keep);
            t.grow(n, keep);
            k0.grow(n, keep);
            k1.grow(n, keep);
        }
        PairBuf buf() { return PairBuf{s.p, t.p, k0.p, k1.p}; }
        void swap(Lists& o)
        {
            s.swap(o.s);
            t.swap(o.t);
            k0.swap(o.k0);
            k1.swap(o.k1);
        }
    };
    Lists cur, nxt, fl, nl;
    cur.alloc(1024);
    nxt.alloc(8192);
    // about 60 far and 30 near pairs per source box on surface point sets
    fl.alloc(std::max<int64_t>(64 * nsb, 1 << 16));
    nl.alloc(std::max<int64_t>(32 * nsb, 1 << 16));
    {
        const int32_t z = 0;
        const uint64_t zk = 0;
        LIST_CUDA(cudaMemcpy(cur.s.p, &z, sizeof(z), cudaMemcpyHostToDevice));
        LIST_CUDA(cudaMemcpy(cur.t.p, &z, sizeof(z), cudaMemcpyHostToDevice));
        LIST_CUDA(cudaMemcpy(cur.k0.p, &zk, sizeof(zk), cudaMemcpyHostToDevice));
        LIST_CUDA(cudaMemcpy(cur.k1.p, &zk, sizeof(zk), cudaMemcpyHostToDevice));
    }
    LBuf<unsigned long long> d_ctr;
    d_ctr.alloc(C_COUNT);
    unsigned long long ctr[C_COUNT] = {0, 0, 0, 0, 0};
    LIST_CUDA(cudaMemcpy(d_ctr.p, ctr, sizeof(ctr), cudaMemcpyHostToDevice));
    long long n_in = 1;
    for (int step = 0; n_in > 0; step++)
    {
        if (step > 42)
            throw Error(2, "interaction lists: walk deeper than the path keys");
        const size_t need_next = (size_t)n_in * 8;
        if (nxt.s.n < need_next)
            nxt.alloc(need_next);
        unsigned long long before[C_COUNT];
        std::copy(ctr, ctr + C_COUNT, before);
        for (;;)
        {
            walk_step_kernel<<<grid_for(n_in), 256>>>(T, cur.buf(), n_in, step, nxt.buf(),
                                                      (long long)nxt.s.n, fl.buf(),
                                                      (long long)fl.s.n, nl.buf(),
                                                      (long long)nl.s.n, d_ctr.p);
            LIST_CUDA(cudaGetLastError());
            LIST_CUDA(cudaMemcpy(ctr, d_ctr.p, sizeof(ctr), cudaMemcpyDeviceToHost));
            if (ctr[C_FAR] <= fl.s.n && ctr[C_NEAR] <= nl.s.n)
                break;
            // outputs overflowed: grow (keeping the earlier steps' pairs), run again
            if (ctr[C_FAR] > fl.s.n)
                fl.grow(2 * ctr[C_FAR], before[C_FAR]);
            if (ctr[C_NEAR] > nl.s.n)
                nl.grow(2 * ctr[C_NEAR], before[C_NEAR]);
            std::copy(before, before + C_COUNT, ctr);
            LIST_CUDA(cudaMemcpy(d_ctr.p, ctr, sizeof(ctr), cudaMemcpyHostToDevice));
        }
        n_in = (long long)ctr[C_NEXT];
        ctr[C_NEXT] = 0;
        LIST_CUDA(cudaMemcpy(d_ctr.p, ctr, sizeof(ctr), cudaMemcpyHostToDevice));
        cur.swap(nxt);
    }
    n_far_pairs = (int64_t)ctr[C_FAR];
    n_near_pairs = (int64_t)ctr[C_NEAR];
    far_target_evals = (int64_t)ctr[C_FAR_EVALS];
    near_point_pairs = (int64_t)ctr[C_NEAR_PAIRS];
    sort_to_csr(fl.buf(), n_far_pairs, nsb, far, far_dev);
    sort_to_csr(nl.buf(), n_near_pairs, nsb, near, near_dev);
    return true;
}

void Plan::ensure_device_pairs()
{
    auto up = [&](const PairLists& L, DevicePairs& dev) {
        const int64_t n = L.off.empty() ? 0 : L.off.back();
        if (dev.n == n && (n == 0 || dev.src))
            return;
        dev = DevicePairs{};
        if (n == 0)
            return;
        std::vector<int32_t> s((size_t)n);
        for (size_t b = 0; b + 1 < L.off.size(); b++)
            std::fill(s.begin() + L.off[b], s.begin() + L.off[b + 1], (int32_t)b);
        LBuf<int32_t> ds, dt;
        ds.alloc(n);
        dt.alloc(n);
        LIST_CUDA(cudaMemcpy(ds.p, s.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
        LIST_CUDA(cudaMemcpy(dt.p, L.tgt.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
        dev.src = device_owned(ds.release());
        dev.tgt = device_owned(dt.release());
        dev.n = n;
    };
    up(far, far_dev);
    up(near, near_dev);
}

} // namespace ifgf
