// Target-leaf lists on the GPU: the per-target view of the source-major
// interaction lists that the evaluation kernels walk (the field-information
// step of computeFieldInfo, octree.hpp:818-880, and the far-target part of
// calculateInterpolationRange, octree.hpp:351-816).  Per target leaf:
//   far  = the far source boxes of the leaf, then of its parent, and so on to
//          the root, each group with sources ascending;
//   near = its near source leaves, ascending.
// Plan::build_target_lists builds the same tables on the host (a plan-only
// init); the two agree entry for entry.
//
//   1. key of every pair = its target box (pairs of source boxes another
//      rank owns get a key past the last box); one stable radix sort by key
//      with the source as value.  The pairs arrive source-ascending, so each
//      target's sources stay ascending.
//   2. per-box offsets by binary search of the sorted keys;
//   3. per leaf, its far count summed over its ancestors and its near count;
//      exclusive scans give the CSR offsets;
//   4. one warp per leaf copies its segments, leaf first.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <climits>

#include "gpu_target_lists.hpp"

namespace ifgf
{
namespace
{

__global__ void tl_keys_kernel(const int32_t* __restrict__ src, const int32_t* __restrict__ tgt,
                               long long n, const int32_t* __restrict__ box_rank, int rank,
                               int ntb, int* __restrict__ keys)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        keys[i] = (rank < 0 || box_rank[src[i]] == rank) ? tgt[i] : ntb;
}

// off[b] = first sorted position with key >= b, for b in [0, ntb]
__global__ void tl_box_offsets_kernel(const int* __restrict__ keys, long long n, int ntb,
                                      long long* __restrict__ off)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > ntb)
        return;
    long long lo = 0, hi = n;
    while (lo < hi)
    {
        const long long mid = (lo + hi) >> 1;
        if (keys[mid] < b)
            lo = mid + 1;
        else
            hi = mid;
    }
    off[b] = lo;
}

// counts of leaf i at i (the entry at nl is 0, so that the exclusive scan's
// last entry is the total)
__global__ void tl_leaf_counts_kernel(const int* __restrict__ leaf_gid, int nl,
                                      const int* __restrict__ parent,
                                      const long long* __restrict__ far_off,
                                      const long long* __restrict__ near_off,
                                      long long* __restrict__ far_cnt,
                                      long long* __restrict__ near_cnt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > nl)
        return;
    if (i == nl)
    {
        far_cnt[i] = near_cnt[i] = 0;
        return;
    }
    const int g = leaf_gid[i];
    long long c = 0;
    for (int a = g; a >= 0; a = parent[a])
        c += far_off[a + 1] - far_off[a];
    far_cnt[i] = c;
    near_cnt[i] = near_off ? near_off[g + 1] - near_off[g] : 0;
}

__global__ void tl_fill_kernel(const int* __restrict__ leaf_gid, int nl,
                               const int* __restrict__ parent,
                               const long long* __restrict__ far_off,
                               const int* __restrict__ far_by_tgt,
                               const long long* __restrict__ near_off,
                               const int* __restrict__ near_by_tgt,
                               const long long* __restrict__ tl_far_off,
                               const long long* __restrict__ tl_near_off,
                               int* __restrict__ tl_far_src, int* __restrict__ tl_near_src)
{
    const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nl)
        return;
    const int g = leaf_gid[w];
    long long o = tl_far_off[w];
    for (int a = g; a >= 0; a = parent[a])
    {
        const long long b = far_off[a], e = far_off[a + 1];
        for (long long j = b + lane; j < e; j += 32)
            tl_far_src[o + (j - b)] = far_by_tgt[j];
        o += e - b;
    }
    if (near_off)
    {
        const long long b = near_off[g], e = near_off[g + 1], q = tl_near_off[w];
        for (long long j = b + lane; j < e; j += 32)
            tl_near_src[q + (j - b)] = near_by_tgt[j];
    }
}

int key_bits(int max_key)
{
    int b = 1;
    while (b < 31 && (1 << b) <= max_key)
        b++;
    return b;
}

// The pairs of `dp` ordered by target box (sources ascending in each), with
// the per-box offsets (ntb + 1 entries).  Another rank's pairs are dropped.
void transpose(const DevicePairs& dp, const DevBuf<int32_t>& box_rank, int rank, int ntb,
               DevBuf<long long>& off, DevBuf<int>& by_tgt)
{
    const long long n = dp.n;
    off.alloc((size_t)ntb + 1);
    if (n == 0)
    {
        off.zero();
        by_tgt.alloc(1);
        return;
    }
    if (n > INT_MAX)
        throw Error(ERR_INVALID, "target-leaf lists: more than 2^31 pairs");
    DevBuf<int> keys, keys_sorted;
    keys.alloc(n);
    keys_sorted.alloc(n);
    by_tgt.alloc(n);
    const unsigned grid = (unsigned)std::min<long long>((n + 255) / 256, 148 * 16);
    tl_keys_kernel<<<grid, 256>>>(dp.src.get(), dp.tgt.get(), n, box_rank.p, rank, ntb, keys.p);
    IFGF_CUDA(cudaGetLastError());
    const int bits = key_bits(ntb);
    size_t tb = 0;
    IFGF_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.p, keys_sorted.p, dp.src.get(),
                                              by_tgt.p, (int)n, 0, bits));
    DevBuf<unsigned char> tmp;
    tmp.alloc(std::max<size_t>(tb, 1));
    IFGF_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.p, keys_sorted.p, dp.src.get(),
                                              by_tgt.p, (int)n, 0, bits));
    tl_box_offsets_kernel<<<(unsigned)((ntb + 1 + 255) / 256), 256>>>(keys_sorted.p, n, ntb,
                                                                        off.p);
    IFGF_CUDA(cudaGetLastError());
}

void exclusive_scan(const DevBuf<long long>& in, DevBuf<long long>& out, int n)
{
    size_t tb = 0;
    IFGF_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, in.p, out.p, n));
    DevBuf<unsigned char> tmp;
    tmp.alloc(std::max<size_t>(tb, 1));
    IFGF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, in.p, out.p, n));
}

} // namespace

void build_target_lists_gpu(Plan& P, int rank, DevBuf<long long>& far_off, DevBuf<int>& far_src,
                            DevBuf<long long>& near_off, DevBuf<int>& near_src)
{
    P.ensure_device_pairs();
    if (P.tleaf_gid.empty())
        P.collect_target_leaves();
    const int64_t ntb64 = P.tgt.num_boxes_total();
    const int64_t nl64 = (int64_t)P.tleaf_gid.size();
    if (ntb64 >= INT_MAX || nl64 >= INT_MAX)
        throw Error(ERR_INVALID, "target-leaf lists: too many target boxes");
    const int ntb = (int)ntb64, nl = (int)nl64;
    DevBuf<int32_t> box_rank;
    if (rank >= 0)
        box_rank.upload(P.box_rank);
    DevBuf<int> parent, leaves;
    parent.upload(P.target_parents());
    {
        std::vector<int> lg(P.tleaf_gid.begin(), P.tleaf_gid.end());
        leaves.upload(lg);
    }
    DevBuf<long long> fbox_off, nbox_off;
    DevBuf<int> far_by_tgt, near_by_tgt;
    transpose(P.far_dev, box_rank, rank, ntb, fbox_off, far_by_tgt);
    transpose(P.near_dev, box_rank, rank, ntb, nbox_off, near_by_tgt);
    DevBuf<long long> fcnt, ncnt;
    fcnt.alloc((size_t)nl + 1);
    ncnt.alloc((size_t)nl + 1);
    tl_leaf_counts_kernel<<<(unsigned)((nl + 1 + 255) / 256), 256>>>(
        leaves.p, nl, parent.p, fbox_off.p, nbox_off.p, fcnt.p, ncnt.p);
    IFGF_CUDA(cudaGetLastError());
    far_off.alloc((size_t)nl + 1);
    near_off.alloc((size_t)nl + 1);
    exclusive_scan(fcnt, far_off, nl + 1);
    exclusive_scan(ncnt, near_off, nl + 1);
    long long tot[2] = {0, 0};
    IFGF_CUDA(cudaMemcpy(&tot[0], far_off.p + nl, sizeof(long long), cudaMemcpyDeviceToHost));
    IFGF_CUDA(cudaMemcpy(&tot[1], near_off.p + nl, sizeof(long long), cudaMemcpyDeviceToHost));
    far_src.alloc((size_t)std::max(tot[0], 1ll));
    near_src.alloc((size_t)std::max(tot[1], 1ll));
    if (nl > 0)
    {
        const long long threads = 32ll * nl;
        tl_fill_kernel<<<(unsigned)((threads + 255) / 256), 256>>>(
            leaves.p, nl, parent.p, fbox_off.p, far_by_tgt.p, nbox_off.p, near_by_tgt.p,
            far_off.p, near_off.p, far_src.p, near_src.p);
        IFGF_CUDA(cudaGetLastError());
    }
    IFGF_CUDA(cudaDeviceSynchronize());
}

} // namespace ifgf
