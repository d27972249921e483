// Octree construction on the GPU (Tree::build_gpu): the steps of Tree::build
// (plan.cpp) as device kernels, with the same arithmetic so that the tree
// matches the host one bit for bit.
//   1. coordinate minima / maxima (block partials, reduced on the host; min
//      and max are exact in any order), inflated on the host;
//   2. the 126-bit Morton key of every point (two 63-bit halves);
//   3. a lexicographic (hi, lo, index) sort as two stable radix sorts (low
//      half, then high half), which keeps equal keys in index order as the
//      host comparator's index tie-break does;
//   4. per level, the children's point ranges of every box to be split by
//      the greedy closed-interval scan (octree.hpp:1139-1170), one warp per
//      box testing 32 consecutive points at a time; the host assembles the
//      levels from these ranges (Tree::make_levels).
// Child bounding boxes use explicitly rounded FP64 operations, so no fused
// multiply-add changes a bound that the host computes without one.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "common.hpp"
#include "plan.hpp"

namespace ifgf
{
namespace
{

#define TREE_CUDA(x)                                                                          \
    do                                                                                         \
    {                                                                                          \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            throw Error(2, std::string("octree build: ") + #x + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T> struct TBuf
{
    T* p = nullptr;
    TBuf() = default;
    TBuf(const TBuf&) = delete;
    TBuf& operator=(const TBuf&) = delete;
    ~TBuf()
    {
        if (p)
            cudaFree(p);
    }
    void alloc(size_t n)
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        TREE_CUDA(cudaMalloc((void**)&p, std::max<size_t>(n, 1) * sizeof(T)));
    }
};

__device__ __forceinline__ uint64_t spread3_dev(uint64_t v)
{
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// coord_code of plan.cpp: sign bit, then |p| * 2^42 in fixed point,
// complemented for negative p
__device__ __forceinline__ uint64_t coord_code_dev(double p)
{
    const uint64_t top = 1ull << 41;
    const bool neg = p < 0.0;
    const double a = __dmul_rn(fabs(p), 4398046511104.0);
    const uint64_t u = a >= (double)(top - 1) ? top - 1 : (uint64_t)a;
    return neg ? (top - 1 - u) : (top | u);
}

struct Vec3
{
    double v[3];
};

__global__ void bbox_partial_kernel(const double* __restrict__ p, long long n, double* part)
{
    __shared__ double smn[3][256], smx[3][256];
    double mn[3], mx[3];
    for (int d = 0; d < 3; d++)
    {
        mn[d] = INFINITY;
        mx[d] = -INFINITY;
    }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        for (int d = 0; d < 3; d++)
        {
            const double x = p[3 * i + d];
            mn[d] = fmin(mn[d], x);
            mx[d] = fmax(mx[d], x);
        }
    for (int d = 0; d < 3; d++)
    {
        smn[d][threadIdx.x] = mn[d];
        smx[d][threadIdx.x] = mx[d];
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1)
    {
        if (threadIdx.x < s)
            for (int d = 0; d < 3; d++)
            {
                smn[d][threadIdx.x] = fmin(smn[d][threadIdx.x], smn[d][threadIdx.x + s]);
                smx[d][threadIdx.x] = fmax(smx[d][threadIdx.x], smx[d][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; d++)
        {
            part[6 * blockIdx.x + d] = smn[d][0];
            part[6 * blockIdx.x + 3 + d] = smx[d][0];
        }
}

// morton_key of plan.cpp: the coordinate normalised as (x - c) / diam
__global__ void morton_keys_kernel(const double* __restrict__ p, long long n, Vec3 c, Vec3 diam,
                                   uint64_t* hi, uint64_t* lo, int* idx)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
    {
        uint64_t k[3];
        for (int d = 0; d < 3; d++)
            k[d] = coord_code_dev(__ddiv_rn(__dsub_rn(p[3 * i + d], c.v[d]), diam.v[d]));
        hi[i] = (spread3_dev(k[2] >> 21) << 2) | (spread3_dev(k[1] >> 21) << 1) |
                spread3_dev(k[0] >> 21);
        lo[i] = (spread3_dev(k[2]) << 2) | (spread3_dev(k[1]) << 1) | spread3_dev(k[0]);
        idx[i] = (int)i;
    }
}

template <typename T>
__global__ void gather_kernel(const T* __restrict__ in, const int* __restrict__ idx, long long n,
                              T* out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = in[idx[i]];
}

__global__ void gather_points_kernel(const double* __restrict__ p, const int* __restrict__ idx,
                                     long long n, double* out)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
    {
        const long long j = idx[i];
        out[3 * i] = p[3 * j];
        out[3 * i + 1] = p[3 * j + 1];
        out[3 * i + 2] = p[3 * j + 2];
    }
}

// One warp per box with more than max_leaf points: for each octant j, the
// first point from the running position on that lies outside child j's
// closed box ends child j (Tree::build's scan, 32 points per step).
__global__ void split_kernel(const double* __restrict__ sp, int nbox,
                             const long long* __restrict__ first,
                             const long long* __restrict__ last,
                             const double* __restrict__ bbmin, const double* __restrict__ bbmax,
                             long long max_leaf, long long* ends)
{
    const int b = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= nbox)
        return;
    const long long f = first[b], l = last[b];
    if (l - f <= max_leaf)
        return;
    long long pidx = f;
    for (int j = 0; j < 8; j++)
    {
        double cmn[3], cmx[3];
        for (int d = 0; d < 3; d++)
        {
            const double size = __dmul_rn(0.5, __dsub_rn(bbmax[3 * b + d], bbmin[3 * b + d]));
            cmn[d] = __dadd_rn(bbmin[3 * b + d], __dmul_rn(size, (double)((j >> d) & 1)));
            cmx[d] = __dadd_rn(cmn[d], size);
        }
        while (pidx < l)
        {
            const long long i = pidx + lane;
            bool stop = i >= l;
            if (!stop)
                for (int d = 0; d < 3; d++)
                {
                    const double x = sp[3 * i + d];
                    stop = stop || !(cmn[d] <= x) || !(x <= cmx[d]);
                }
            const unsigned m = __ballot_sync(0xffffffffu, stop);
            if (m)
            {
                pidx += __ffs(m) - 1;
                break;
            }
            pidx += 32;
        }
        if (lane == 0)
            ends[8 * (long long)b + j] = pidx;
    }
}

unsigned grid_for(long long n, int threads)
{
    return (unsigned)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148 * 8));
}

} // namespace

void Tree::build_gpu(const double* p, int64_t n_pts, int64_t leaf_size)
{
    n = n_pts;
    max_leaf = leaf_size;
    if (n < 1 || n > (int64_t)0x7fffffff)
        throw Error(1, "octree build: point count out of range");
    TBuf<double> dp, dsp;
    dp.alloc(3 * (size_t)n);
    TREE_CUDA(cudaMemcpy(dp.p, p, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    // 1. bounding box
    const int bt = 256;
    const unsigned nb = grid_for(n, bt);
    TBuf<double> part;
    part.alloc(6 * (size_t)nb);
    bbox_partial_kernel<<<nb, bt>>>(dp.p, n, part.p);
    TREE_CUDA(cudaGetLastError());
    std::vector<double> hp(6 * (size_t)nb);
    TREE_CUDA(cudaMemcpy(hp.data(), part.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost));
    double mn[3], mx[3];
    for (int d = 0; d < 3; d++)
    {
        mn[d] = hp[d];
        mx[d] = hp[3 + d];
    }
    for (unsigned q = 1; q < nb; q++)
        for (int d = 0; d < 3; d++)
        {
            mn[d] = std::min(mn[d], hp[6 * q + d]);
            mx[d] = std::max(mx[d], hp[6 * q + 3 + d]);
        }
    inflate_bbox(mn, mx);
    Vec3 c, diam;
    for (int d = 0; d < 3; d++)
    {
        c.v[d] = (mx[d] + mn[d]) / 2.0;
        diam.v[d] = mx[d] - mn[d];
    }
    // 2. keys, 3. stable sorts: by the low half, then by the high half
    TBuf<uint64_t> hi, lo, hi2, lo2;
    TBuf<int> idx, idx2;
    hi.alloc(n);
    lo.alloc(n);
    hi2.alloc(n);
    lo2.alloc(n);
    idx.alloc(n);
    idx2.alloc(n);
    morton_keys_kernel<<<grid_for(n, bt), bt>>>(dp.p, n, c, diam, hi.p, lo.p, idx.p);
    TREE_CUDA(cudaGetLastError());
    size_t tb1 = 0, tb2 = 0;
    TREE_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb1, lo.p, lo2.p, idx.p, idx2.p, (int)n, 0,
                                              63));
    TREE_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb2, hi2.p, hi.p, idx2.p, idx.p, (int)n, 0,
                                              63));
    TBuf<unsigned char> tmp;
    tmp.alloc(std::max(tb1, tb2));
    size_t tb = std::max(tb1, tb2);
    TREE_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, lo.p, lo2.p, idx.p, idx2.p, (int)n, 0, 63));
    gather_kernel<uint64_t><<<grid_for(n, bt), bt>>>(hi.p, idx2.p, n, hi2.p);
    TREE_CUDA(cudaGetLastError());
    tb = std::max(tb1, tb2);
    TREE_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, hi2.p, hi.p, idx2.p, idx.p, (int)n, 0, 63));
    std::vector<int> hidx(n);
    TREE_CUDA(cudaMemcpy(hidx.data(), idx.p, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost));
    perm.assign(hidx.begin(), hidx.end());
    dsp.alloc(3 * (size_t)n);
    gather_points_kernel<<<grid_for(n, bt), bt>>>(dp.p, idx.p, n, dsp.p);
    TREE_CUDA(cudaGetLastError());
    pts.resize(3 * (size_t)n);
    TREE_CUDA(cudaMemcpy(pts.data(), dsp.p, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    // 4. levels: children's ranges of each level on the device
    TBuf<long long> dfirst, dlast, dends;
    TBuf<double> dbmin, dbmax;
    make_levels(mn, mx, [&](const TreeLevel& L, std::vector<int64_t>& ends) {
        const int nbox = (int)L.size();
        bool any = false;
        for (int b = 0; b < nbox && !any; b++)
            any = L.last[b] - L.first[b] > max_leaf;
        if (!any)
            return;
        dfirst.alloc(nbox);
        dlast.alloc(nbox);
        dbmin.alloc(3 * (size_t)nbox);
        dbmax.alloc(3 * (size_t)nbox);
        dends.alloc(8 * (size_t)nbox);
        static_assert(sizeof(long long) == sizeof(int64_t), "64-bit ranges");
        TREE_CUDA(cudaMemcpy(dfirst.p, L.first.data(), nbox * sizeof(long long), cudaMemcpyHostToDevice));
        TREE_CUDA(cudaMemcpy(dlast.p, L.last.data(), nbox * sizeof(long long), cudaMemcpyHostToDevice));
        TREE_CUDA(cudaMemcpy(dbmin.p, L.bbmin.data(), 3 * (size_t)nbox * sizeof(double),
                             cudaMemcpyHostToDevice));
        TREE_CUDA(cudaMemcpy(dbmax.p, L.bbmax.data(), 3 * (size_t)nbox * sizeof(double),
                             cudaMemcpyHostToDevice));
        TREE_CUDA(cudaMemset(dends.p, 0xff, 8 * (size_t)nbox * sizeof(long long)));
        const int wt = 256; // 8 warps, one box each
        const unsigned grid = (unsigned)((nbox + wt / 32 - 1) / (wt / 32));
        split_kernel<<<grid, wt>>>(dsp.p, nbox, dfirst.p, dlast.p, dbmin.p, dbmax.p, max_leaf,
                                   dends.p);
        TREE_CUDA(cudaGetLastError());
        TREE_CUDA(cudaMemcpy(ends.data(), dends.p, 8 * (size_t)nbox * sizeof(long long),
                             cudaMemcpyDeviceToHost));
    });
}

} // namespace ifgf
