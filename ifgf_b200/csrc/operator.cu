// IFGF operator: device tables and the per-level CUDA pipeline for sm_100a.
//
// mult (IfgfOperator::mult, ifgfoperator.hpp:246-867) runs level-synchronously
// from the deepest source level to the root.  Per level:
//   coarse_values  -- nodal values of every active coarse cone: leaves sample
//                     the factored kernel (evaluateFactoredKernel), other
//                     boxes sum their children's fine interpolants at the
//                     cone's Chebyshev nodes times the centre-shift factor
//                     (transferInterp + transfer_factor);
//   coarse_to_fine -- coarse nodal values -> fine Chebyshev coefficients of the
//                     active sub-cones (chebtransform, coarseToFine and the
//                     second chebtransform folded into three small matrices).
// Then one target_eval launch per target leaf adds the near field (direct
// sums over neighbouring source leaves) and the far field (fine interpolants
// of every admissible source box times the centred factor CF) and writes the
// result in the caller's order.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <sstream>

#include "device_math.cuh"
#include "operator.hpp"

namespace ifgf
{

static constexpr int ERR_INVALID = 1, ERR_CUDA = 2, ERR_STATE = 3, ERR_OOM = 4;

#define IFGF_CUDA(x)                                                                          \
    do                                                                                         \
    {                                                                                          \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            throw Error(ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));           \
    } while (0)

template <typename T> struct DevBuf
{
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n)
    {
        o.p = nullptr;
        o.n = 0;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count)
    {
        release();
        if (count == 0)
            return;
        cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
        if (e != cudaSuccess)
        {
            cudaGetLastError();
            p = nullptr;
            throw Error(ERR_OOM, "cudaMalloc(" + std::to_string(count * sizeof(T)) +
                                     " bytes) failed: " + cudaGetErrorString(e));
        }
        n = count;
    }
    void upload(const T* h, size_t count)
    {
        alloc(count);
        if (count)
            IFGF_CUDA(cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice));
    }
    void upload(const std::vector<T>& v) { upload(v.data(), v.size()); }
    void zero()
    {
        if (n)
            IFGF_CUDA(cudaMemset(p, 0, n * sizeof(T)));
    }
    void release()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

struct DeviceState
{
    DevBuf<LevelGeom> lv;
    DevBuf<double> box_c, box_H;
    DevBuf<int> box_first, box_last, box_child, box_level;
    DevBuf<unsigned char> box_leaf;
    DevBuf<double> sx, sy, sz, nx, ny, nz, tx, ty, tz;
    DevBuf<long long> src_perm, tgt_perm;
    std::vector<DevBuf<int>> cc_box, cc_el, fc_box, fc_el; // per level
    DevBuf<int> fmap;
    DevBuf<double> hi_nodes, A;
    DevBuf<int> tl_first, tl_last, tl_far_src, tl_near_src;
    DevBuf<long long> tl_far_off, tl_near_off;
    DevBuf<double2> w, cvals, fcoef;
    DevBuf<unsigned long long> err;
    DevBuf<double> io_w, io_u; // staging for host-buffer mult
    std::vector<cudaEvent_t> prof_ev;
    int n_tleaf = 0;
    size_t c2f_smem = 0;
    int cv_threads = 0;
    ~DeviceState()
    {
        for (auto& e : prof_ev)
            cudaEventDestroy(e);
    }
};

// ---------------------------------------------------------------------------
// Kernel arguments
// ---------------------------------------------------------------------------
struct TreeArgs
{
    const double* __restrict__ box_c;
    const double* __restrict__ box_H;
    const int* __restrict__ box_first;
    const int* __restrict__ box_last;
    const int* __restrict__ box_child;
    const int* __restrict__ box_level;
    const unsigned char* __restrict__ box_leaf;
};

struct SrcArgs
{
    const double* __restrict__ sx;
    const double* __restrict__ sy;
    const double* __restrict__ sz;
    const double* __restrict__ nx;
    const double* __restrict__ ny;
    const double* __restrict__ nz;
};

// ---------------------------------------------------------------------------
// Setup kernels: active-cone marking (octree.hpp:571-690) and compaction
// ---------------------------------------------------------------------------
// One CTA per far pair (source box, target range): mark the fine and coarse
// cones that contain the far targets (octree.hpp:574-590).
__global__ void mark_far_kernel(LevelGeom G, TreeArgs T, const int* __restrict__ fp_src,
                                const int* __restrict__ fp_t0, const int* __restrict__ fp_t1,
                                const double* __restrict__ tx, const double* __restrict__ ty,
                                const double* __restrict__ tz, int* fmark, int* cmark)
{
    const int pr = blockIdx.x;
    const int sb = fp_src[pr];
    const int lb = sb - G.box_off;
    const double xc0 = T.box_c[3 * sb], xc1 = T.box_c[3 * sb + 1], xc2 = T.box_c[3 * sb + 2];
    const double H = T.box_H[sb];
    const long long nf = (long long)G.nf[0] * G.nf[1] * G.nf[2];
    const long long nc = (long long)G.nc[0] * G.nc[1] * G.nc[2];
    const int t1 = fp_t1[pr];
    for (int t = fp_t0[pr] + threadIdx.x; t < t1; t += blockDim.x)
    {
        double s[3];
        cart_to_interp(tx[t] - xc0, ty[t] - xc1, tz[t] - xc2, H, s);
        const int fe = element_for_point(s, G.dmin, G.dmax, G.hf, G.nf);
        const int ce = element_for_point(s, G.dmin, G.dmax, G.hc, G.nc);
        if (fe >= 0)
            fmark[G.fmap_off + lb * nf + fe] = 1;
        if (ce >= 0)
            cmark[lb * nc + ce] = 1;
    }
}

// One CTA per active coarse cone of the parent level: map the cone's
// Chebyshev nodes into each child's frame and mark the child cones that
// contain them (TwoGrid branch, octree.hpp:660-690).
__global__ void mark_parent_kernel(LevelGeom PG, LevelGeom G, TreeArgs T,
                                   const int* __restrict__ pcc_box,
                                   const int* __restrict__ pcc_el,
                                   const double* __restrict__ hi_nodes, int P_hi, int* fmark,
                                   int* cmark)
{
    const int c = blockIdx.x;
    const int pb = pcc_box[c], pel = pcc_el[c];
    const double pxc[3] = {T.box_c[3 * pb], T.box_c[3 * pb + 1], T.box_c[3 * pb + 2]};
    const double pH = T.box_H[pb];
    const long long nf = (long long)G.nf[0] * G.nf[1] * G.nf[2];
    const long long nc = (long long)G.nc[0] * G.nc[1] * G.nc[2];
    for (int n = threadIdx.x; n < P_hi; n += blockDim.x)
    {
        double loc[3] = {hi_nodes[3 * n], hi_nodes[3 * n + 1], hi_nodes[3 * n + 2]};
        double s[3], x[3];
        from_local(pel, loc, PG.dmin, PG.hc, PG.nc, s);
        interp_to_cart(s, pxc, pH, x);
        for (int o = 0; o < 8; o++)
        {
            const int cb = T.box_child[8 * pb + o];
            if (cb < 0)
                continue;
            const int lb = cb - G.box_off;
            double s2[3];
            cart_to_interp(x[0] - T.box_c[3 * cb], x[1] - T.box_c[3 * cb + 1],
                           x[2] - T.box_c[3 * cb + 2], T.box_H[cb], s2);
            const int fe = element_for_point(s2, G.dmin, G.dmax, G.hf, G.nf);
            const int ce = element_for_point(s2, G.dmin, G.dmax, G.hc, G.nc);
            if (fe >= 0)
                fmark[G.fmap_off + lb * nf + fe] = 1;
            if (ce >= 0)
                cmark[lb * nc + ce] = 1;
        }
    }
}

// mark -> global index (or -1); emits (box, element) lists in (box, element)
// order.
__global__ void finalize_map_kernel(int* map, const int* __restrict__ idx, long long n, int n_el,
                                    int box_off, int gbase, int* list_box, int* list_el)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
    {
        if (map[i])
        {
            const int k = idx[i];
            list_box[k] = box_off + (int)(i / n_el);
            list_el[k] = (int)(i % n_el);
            map[i] = gbase + k;
        }
        else
        {
            map[i] = -1;
        }
    }
}

// ---------------------------------------------------------------------------
// mult kernels
// ---------------------------------------------------------------------------
__global__ void permute_weights_kernel(const double* __restrict__ in, int real_in,
                                       const long long* __restrict__ perm, double2* w,
                                       long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
    {
        const long long j = perm[i];
        w[i] = real_in ? make_double2(in[j], 0.0) : reinterpret_cast<const double2*>(in)[j];
    }
}

struct CoarseArgs
{
    LevelGeom G;  // this level
    LevelGeom GC; // child level (valid when the level has children)
    TreeArgs T;
    SrcArgs S;
    const int* __restrict__ cc_box;
    const int* __restrict__ cc_el;
    const double* __restrict__ hi_nodes;
    const double2* __restrict__ w;
    const int* __restrict__ fmap;
    const double2* __restrict__ fcoef;
    double2* cvals;
    unsigned long long* err;
    int P_hi, P_lo;
    int lo[3];
    KParams kp;
};

constexpr int CV_MAXNPT = 4; // nodes per thread

// Nodal values of one active coarse cone per CTA.
template <int KIND>
__global__ void __launch_bounds__(512) coarse_values_kernel(CoarseArgs a)
{
    using P = Plugin<KIND>;
    extern __shared__ double sm[];
    const int c = blockIdx.x;
    const int box = a.cc_box[c], el = a.cc_el[c];
    const double xc[3] = {a.T.box_c[3 * box], a.T.box_c[3 * box + 1], a.T.box_c[3 * box + 2]};
    const double H = a.T.box_H[box];
    const bool leaf = a.T.box_leaf[box];

    double y[CV_MAXNPT][3];
    double dc[CV_MAXNPT];
    cplx<double> acc[CV_MAXNPT];
#pragma unroll
    for (int q = 0; q < CV_MAXNPT; q++)
    {
        const int n = threadIdx.x + q * blockDim.x;
        acc[q] = {0.0, 0.0};
        dc[q] = 0;
        y[q][0] = y[q][1] = y[q][2] = 0;
        if (n < a.P_hi)
        {
            const double loc[3] = {a.hi_nodes[3 * n], a.hi_nodes[3 * n + 1], a.hi_nodes[3 * n + 2]};
            double s[3];
            from_local(el, loc, a.G.dmin, a.G.hc, a.G.nc, s);
            interp_to_cart(s, xc, H, y[q]);
            const double e0 = y[q][0] - xc[0], e1 = y[q][1] - xc[1], e2 = y[q][2] - xc[2];
            dc[q] = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
        }
    }

    if (leaf)
    {
        // evaluateFactoredKernel over the leaf's sources, staged in shared memory
        const int nt = blockDim.x;
        double* xs = sm;
        double* ys = xs + nt;
        double* zs = ys + nt;
        double* wr = zs + nt;
        double* wi = wr + nt;
        double* n0 = wi + nt;
        double* n1 = n0 + nt;
        double* n2 = n1 + nt;
        const int f = a.T.box_first[box], l = a.T.box_last[box];
        for (int cs = f; cs < l; cs += nt)
        {
            const int cnt = min(nt, l - cs);
            __syncthreads();
            if (threadIdx.x < cnt)
            {
                const int i = cs + threadIdx.x;
                xs[threadIdx.x] = a.S.sx[i];
                ys[threadIdx.x] = a.S.sy[i];
                zs[threadIdx.x] = a.S.sz[i];
                const double2 wv = a.w[i];
                wr[threadIdx.x] = wv.x;
                wi[threadIdx.x] = wv.y;
                if (P::needs_normals)
                {
                    n0[threadIdx.x] = a.S.nx[i];
                    n1[threadIdx.x] = a.S.ny[i];
                    n2[threadIdx.x] = a.S.nz[i];
                }
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < CV_MAXNPT; q++)
            {
                const int n = threadIdx.x + q * blockDim.x;
                if (n >= a.P_hi)
                    continue;
                for (int i = 0; i < cnt; i++)
                {
                    const double av[3] = {xs[i] - y[q][0], ys[i] - y[q][1], zs[i] - y[q][2]};
                    const double nv[3] = {P::needs_normals ? n0[i] : 0.0,
                                          P::needs_normals ? n1[i] : 0.0,
                                          P::needs_normals ? n2[i] : 0.0};
                    const cplx<double> v = P::factored(av, nv, {wr[i], wi[i]}, y[q], dc[q], a.kp);
                    acc[q] = cadd(acc[q], v);
                }
            }
        }
    }
    else
    {
        // transferInterp from every child's fine interpolant
        const LevelGeom& C = a.GC;
        const long long nf = (long long)C.nf[0] * C.nf[1] * C.nf[2];
        for (int o = 0; o < 8; o++)
        {
            const int cb = a.T.box_child[8 * box + o];
            if (cb < 0)
                continue;
            const double cxc[3] = {a.T.box_c[3 * cb], a.T.box_c[3 * cb + 1], a.T.box_c[3 * cb + 2]};
            const double cH = a.T.box_H[cb];
            const int* fm = a.fmap + C.fmap_off + (long long)(cb - C.box_off) * nf;
#pragma unroll
            for (int q = 0; q < CV_MAXNPT; q++)
            {
                const int n = threadIdx.x + q * blockDim.x;
                if (n >= a.P_hi)
                    continue;
                const double p0 = y[q][0] - cxc[0], p1 = y[q][1] - cxc[1], p2 = y[q][2] - cxc[2];
                double s[3], loc[3];
                cart_to_interp(p0, p1, p2, cH, s);
                const int fe = element_for_point(s, C.dmin, C.dmax, C.hf, C.nf);
                if (fe < 0)
                    continue;
                const int gf = fm[fe];
                if (gf < 0)
                {
                    atomicAdd(a.err, 1ull);
                    continue;
                }
                to_local(fe, s, C.dmin, C.hf, C.nf, loc);
                const cplx<double> v =
                    cheb_eval3<16>(a.fcoef + (size_t)gf * a.P_lo, loc, a.lo);
                const double e0 = y[q][0] - xc[0], e1 = y[q][1] - xc[1], e2 = y[q][2] - xc[2];
                const cplx<double> tf =
                    P::transfer(p0 * p0 + p1 * p1 + p2 * p2, e0 * e0 + e1 * e1 + e2 * e2, a.kp);
                acc[q] = cadd(acc[q], cmul(v, tf));
            }
        }
    }
#pragma unroll
    for (int q = 0; q < CV_MAXNPT; q++)
    {
        const int n = threadIdx.x + q * blockDim.x;
        if (n < a.P_hi)
            a.cvals[(size_t)c * a.P_hi + n] = make_double2(acc[q].re, acc[q].im);
    }
}

struct C2FArgs
{
    LevelGeom G;
    const int* __restrict__ cc_box;
    const int* __restrict__ cc_el;
    const double2* __restrict__ cvals;
    const double* __restrict__ A; // A0 | A1 | A2, row-major (f_d lo_d) x ho_d
    const int* __restrict__ fmap;
    double2* fcoef;
    int hi[3], lo[3], f[3];
    int P_hi, P_lo;
};

// Coarse nodal values -> fine Chebyshev coefficients of the active sub-cones
// (chebtransform chebinterp.hpp:176-250, coarseToFine ifgfoperator.hpp:1539-1637
// and the fine chebtransform :1115-1124, composed per dimension).
__global__ void __launch_bounds__(256) coarse_to_fine_kernel(C2FArgs a)
{
    extern __shared__ double2 s2[];
    const int c = blockIdx.x;
    const int box = a.cc_box[c], el = a.cc_el[c];
    const int h0 = a.hi[0], h1 = a.hi[1], h2 = a.hi[2];
    const int F0 = a.f[0] * a.lo[0], F1 = a.f[1] * a.lo[1];
    const int sz0 = a.P_hi;
    const int sz2 = max(F0 * h1 * h2, F0 * F1 * a.lo[2]);
    double2* B0 = s2;
    double2* B2 = B0 + sz0;
    double2* B1 = B2 + sz2;
    const double* A0 = a.A;
    const double* A1 = A0 + F0 * h0;
    const double* A2 = A1 + F1 * h1;

    for (int i = threadIdx.x; i < sz0; i += blockDim.x)
        B0[i] = a.cvals[(size_t)c * a.P_hi + i];
    __syncthreads();
    // mode 0
    for (int o = threadIdx.x; o < F0 * h1 * h2; o += blockDim.x)
    {
        const int i0 = o % F0, r = o / F0; // r = m1 + h1 m2
        double re = 0, im = 0;
        for (int m = 0; m < h0; m++)
        {
            const double av = A0[i0 * h0 + m];
            const double2 v = B0[m + h0 * r];
            re = fma(av, v.x, re);
            im = fma(av, v.y, im);
        }
        B2[o] = make_double2(re, im);
    }
    __syncthreads();
    // mode 1
    for (int o = threadIdx.x; o < F0 * F1 * h2; o += blockDim.x)
    {
        const int i0 = o % F0, r = o / F0;
        const int i1 = r % F1, m2 = r / F1;
        double re = 0, im = 0;
        for (int m = 0; m < h1; m++)
        {
            const double av = A1[i1 * h1 + m];
            const double2 v = B2[i0 + F0 * (m + h1 * m2)];
            re = fma(av, v.x, re);
            im = fma(av, v.y, im);
        }
        B1[o] = make_double2(re, im);
    }
    const int nc0 = a.G.nc[0], nc1 = a.G.nc[1];
    const int hid0 = el % nc0, hid1 = (el / nc0) % nc1, hid2 = el / (nc0 * nc1);
    const int nf0 = a.G.nf[0], nf1 = a.G.nf[1];
    const long long nft = (long long)nf0 * nf1 * a.G.nf[2];
    const int* fm = a.fmap + a.G.fmap_off + (long long)(box - a.G.box_off) * nft;
    const int lo0 = a.lo[0], lo1 = a.lo[1], lo2 = a.lo[2];
    for (int j2 = 0; j2 < a.f[2]; j2++)
    {
        __syncthreads();
        // mode 2, rows j2*lo2 .. j2*lo2+lo2-1
        for (int o = threadIdx.x; o < F0 * F1 * lo2; o += blockDim.x)
        {
            const int i01 = o % (F0 * F1), i2 = o / (F0 * F1);
            const int row = j2 * lo2 + i2;
            double re = 0, im = 0;
            for (int m = 0; m < h2; m++)
            {
                const double av = A2[row * h2 + m];
                const double2 v = B1[i01 + F0 * F1 * m];
                re = fma(av, v.x, re);
                im = fma(av, v.y, im);
            }
            B2[o] = make_double2(re, im);
        }
        __syncthreads();
        // scatter the f0 x f1 sub-cones of this slice
        const int nsub = a.f[0] * a.f[1];
        for (int o = threadIdx.x; o < nsub * a.P_lo; o += blockDim.x)
        {
            const int sub = o / a.P_lo, q = o % a.P_lo;
            const int j0 = sub % a.f[0], j1 = sub / a.f[0];
            const int fel = ((hid2 * a.f[2] + j2) * nf1 + (hid1 * a.f[1] + j1)) * nf0 +
                            (hid0 * a.f[0] + j0);
            const int gf = fm[fel];
            if (gf < 0)
                continue;
            const int i0 = q % lo0, i1 = (q / lo0) % lo1, i2 = q / (lo0 * lo1);
            a.fcoef[(size_t)gf * a.P_lo + q] =
                B2[(j0 * lo0 + i0) + F0 * ((j1 * lo1 + i1) + F1 * i2)];
        }
    }
}

struct EvalArgs
{
    const LevelGeom* __restrict__ lv;
    TreeArgs T;
    SrcArgs S;
    const double* __restrict__ tx;
    const double* __restrict__ ty;
    const double* __restrict__ tz;
    const long long* __restrict__ tgt_perm;
    const int* __restrict__ tl_first;
    const int* __restrict__ tl_last;
    const long long* __restrict__ far_off;
    const int* __restrict__ far_src;
    const long long* __restrict__ near_off;
    const int* __restrict__ near_src;
    const double2* __restrict__ w;
    const int* __restrict__ fmap;
    const double2* __restrict__ fcoef;
    double* out; // complex (interleaved) or real for Laplace
    int real_out;
    unsigned long long* err;
    int P_lo;
    int lo[3];
    KParams kp;
};

constexpr int EVAL_THREADS = 128;

// One CTA per target leaf: near field + far field, written in caller order.
template <int KIND>
__global__ void __launch_bounds__(EVAL_THREADS) target_eval_kernel(EvalArgs a)
{
    using P = Plugin<KIND>;
    __shared__ double xs[EVAL_THREADS], ys[EVAL_THREADS], zs[EVAL_THREADS];
    __shared__ double wr[EVAL_THREADS], wi[EVAL_THREADS];
    __shared__ double n0[P::needs_normals ? EVAL_THREADS : 1], n1[P::needs_normals ? EVAL_THREADS : 1],
        n2[P::needs_normals ? EVAL_THREADS : 1];
    const int tl = blockIdx.x;
    const int tf = a.tl_first[tl], tlast = a.tl_last[tl];
    const long long nb0 = a.near_off[tl], nb1 = a.near_off[tl + 1];
    const long long fb0 = a.far_off[tl], fb1 = a.far_off[tl + 1];
    for (int base = tf; base < tlast; base += EVAL_THREADS)
    {
        const int t = base + threadIdx.x;
        const bool valid = t < tlast;
        const double y0 = valid ? a.tx[t] : 0.0, y1 = valid ? a.ty[t] : 0.0,
                     y2 = valid ? a.tz[t] : 0.0;
        cplx<double> acc = {0.0, 0.0};
        // near field (evaluateNearField, ifgfoperator.hpp:900-960)
        for (long long e = nb0; e < nb1; e++)
        {
            const int sb = a.near_src[e];
            const int sf = a.T.box_first[sb], sl = a.T.box_last[sb];
            for (int cs = sf; cs < sl; cs += EVAL_THREADS)
            {
                const int cnt = min(EVAL_THREADS, sl - cs);
                __syncthreads();
                if (threadIdx.x < cnt)
                {
                    const int i = cs + threadIdx.x;
                    xs[threadIdx.x] = a.S.sx[i];
                    ys[threadIdx.x] = a.S.sy[i];
                    zs[threadIdx.x] = a.S.sz[i];
                    const double2 wv = a.w[i];
                    wr[threadIdx.x] = wv.x;
                    wi[threadIdx.x] = wv.y;
                    if (P::needs_normals)
                    {
                        n0[threadIdx.x] = a.S.nx[i];
                        n1[threadIdx.x] = a.S.ny[i];
                        n2[threadIdx.x] = a.S.nz[i];
                    }
                }
                __syncthreads();
                if (valid)
                {
                    for (int i = 0; i < cnt; i++)
                    {
                        const double x[3] = {xs[i] - y0, ys[i] - y1, zs[i] - y2};
                        const double nv[3] = {P::needs_normals ? n0[i] : 0.0,
                                              P::needs_normals ? n1[i] : 0.0,
                                              P::needs_normals ? n2[i] : 0.0};
                        const cplx<double> g = P::kernel(x, nv, a.kp);
                        cfma(acc, cplx<double>{wr[i], wi[i]}, g);
                    }
                }
            }
        }
        // far field (evaluateFarField / evaluateFromInterp, ifgfoperator.hpp:963-1012, 1736-1891)
        if (valid)
        {
            for (long long e = fb0; e < fb1; e++)
            {
                const int sb = a.far_src[e];
                const LevelGeom& G = a.lv[a.T.box_level[sb]];
                const double p[3] = {y0 - a.T.box_c[3 * sb], y1 - a.T.box_c[3 * sb + 1],
                                     y2 - a.T.box_c[3 * sb + 2]};
                double s[3], loc[3];
                cart_to_interp(p[0], p[1], p[2], a.T.box_H[sb], s);
                const int fe = element_for_point(s, G.dmin, G.dmax, G.hf, G.nf);
                if (fe < 0)
                    continue;
                const long long nft = (long long)G.nf[0] * G.nf[1] * G.nf[2];
                const int gf = a.fmap[G.fmap_off + (long long)(sb - G.box_off) * nft + fe];
                if (gf < 0)
                {
                    atomicAdd(a.err, 1ull);
                    continue;
                }
                to_local(fe, s, G.dmin, G.hf, G.nf, loc);
                const cplx<double> v = cheb_eval3<16>(a.fcoef + (size_t)gf * a.P_lo, loc, a.lo);
                cfma(acc, v, P::cf(p, a.kp));
            }
            const long long o = a.tgt_perm[t];
            if (a.real_out)
                a.out[o] = acc.re;
            else
            {
                a.out[2 * o] = acc.re;
                a.out[2 * o + 1] = acc.im;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static std::vector<double> cheb_nodes(int n) // chebinterp.hpp:26-39
{
    std::vector<double> v(n);
    for (int i = 0; i < n; i++)
        v[i] = std::cos((2. * i + 1.0) / (2. * n) * M_PI);
    return v;
}

// Per-dimension composition of chebtransform (ho), evaluation at the f
// sub-interval node sets and chebtransform (lo): (f lo) x ho, row-major.
static std::vector<double> c2f_matrix(int ho, int lo, int f)
{
    std::vector<long double> Tc((size_t)ho * ho), E((size_t)f * lo * ho), Tf((size_t)lo * lo);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < ho; m++)
        for (int s = 0; s < ho; s++)
            Tc[(size_t)m * ho + s] =
                (m == 0 ? 1.0L : 2.0L) / ho * std::cos(m * pi * (2.0L * s + 1.0L) / (2.0L * ho));
    for (int q = 0; q < lo; q++)
        for (int i = 0; i < lo; i++)
            Tf[(size_t)q * lo + i] =
                (q == 0 ? 1.0L : 2.0L) / lo * std::cos(q * pi * (2.0L * i + 1.0L) / (2.0L * lo));
    for (int j = 0; j < f; j++)
    {
        const long double mn = -1.0L + j * (2.0L / f), mx = mn + 2.0L / f;
        const long double A = 0.5L * (mx - mn), B = 0.5L * (mx + mn);
        for (int i = 0; i < lo; i++)
        {
            const long double x = std::cos((2.0L * i + 1.0L) / (2.0L * lo) * pi) * A + B;
            long double t0 = 1, t1 = x;
            for (int m = 0; m < ho; m++)
            {
                long double tm = m == 0 ? 1.0L : (m == 1 ? x : 2 * x * t1 - t0);
                if (m >= 2)
                {
                    t0 = t1;
                    t1 = tm;
                }
                E[((size_t)j * lo + i) * ho + m] = tm;
            }
        }
    }
    std::vector<double> out((size_t)f * lo * ho);
    for (int j = 0; j < f; j++)
        for (int q = 0; q < lo; q++)
            for (int s = 0; s < ho; s++)
            {
                long double acc = 0;
                for (int i = 0; i < lo; i++)
                {
                    long double e = 0;
                    for (int m = 0; m < ho; m++)
                        e += E[((size_t)j * lo + i) * ho + m] * Tc[(size_t)m * ho + s];
                    acc += Tf[(size_t)q * lo + i] * e;
                }
                out[((size_t)j * lo + q) * ho + s] = (double)acc;
            }
    return out;
}

Operator::Operator(int kind, double k_re, double k_im, int64_t leaf_size, int64_t order,
                   int64_t n_elem, double tol)
    : kind_(kind), kr_(k_re), ki_(k_im), tol_(tol), leaf_(leaf_size), order0_((int)order)
{
    if (kind < K_LAPLACE || kind > K_COMBINEDFIELD)
        throw Error(ERR_INVALID, "unknown kernel kind " + std::to_string(kind));
    if (leaf_size < 1)
        throw Error(ERR_INVALID, "leaf size must be >= 1");
    if (order < 1 || order > 24)
        throw Error(ERR_INVALID, "order must be in [1, 24]");
    if (n_elem < 1)
        throw Error(ERR_INVALID, "n_elements must be >= 1");
    if (!std::isfinite(k_re) || !std::isfinite(k_im))
        throw Error(ERR_INVALID, "wavenumber must be finite");
    base_n_[0] = 1 * n_elem; // ifgfoperator.hpp:40-51
    base_n_[1] = 2 * n_elem;
    base_n_[2] = 4 * n_elem;
    for (int i = 0; i < 3; i++)
        base_order_[i] = (int)order;
    dev_.reset(new DeviceState());
}

Operator::~Operator() = default;

void Operator::set_dx(int dx)
{
    if (dx < -1 || dx > 2)
        throw Error(ERR_INVALID, "dx must be -1, 0, 1 or 2");
    dx_ = dx;
}

void Operator::set_precision(int mode)
{
    if (mode != PREC_FP64 && mode != PREC_MIXED)
        throw Error(ERR_INVALID, "precision must be FP64 (0) or MIXED (1)");
    precision_ = mode;
}

// orderForBox of each plug-in (helmholtz_ifgf.hpp:158-170, laplace_ifgf.hpp:134-146,
// modified_helmholtz_ifgf.hpp:138-153, grad_helmholtz_ifgf.hpp:238-266,
// double_layer_helmholtz_ifgf.hpp:161-188, combined_field_helmholtz_ifgf.hpp:184-199)
void Operator::order_for_box(int step, int* out) const
{
    for (int i = 0; i < 3; i++)
    {
        out[i] = base_order_[i];
        if (step == 0)
        {
            out[i] = base_order_[i] - 3;
            if (kind_ == K_HELMHOLTZ || kind_ == K_GRADHELMHOLTZ)
                out[i] = std::max(out[i], 2);
        }
    }
}

// elementsForBox of each plug-in (helmholtz_ifgf.hpp:172-195, laplace_ifgf.hpp:148-158,
// modified_helmholtz_ifgf.hpp:155-185, grad_helmholtz_ifgf.hpp:268-292,
// double_layer_helmholtz_ifgf.hpp:190-214, combined_field_helmholtz_ifgf.hpp:201-224)
void Operator::elements_for_box(double H, int step, int64_t* out) const
{
    int64_t base[3] = {base_n_[0], base_n_[1], base_n_[2]};
    if (kind_ == K_LAPLACE)
    {
        for (int i = 0; i < 3; i++)
            out[i] = step == 0 ? base[i] * 3 : base[i];
        return;
    }
    if (step == 0 && kind_ != K_MODHELMHOLTZ)
        for (int i = 0; i < 3; i++)
            base[i] *= 3;
    for (int i = 0; i < 3; i++)
    {
        int64_t c;
        if (kind_ == K_MODHELMHOLTZ)
        {
            const int delta = (int)std::ceil(std::max(std::abs(ki_) * H / (2 * (2 + kr_)), 1.0));
            c = (int64_t)std::ceil((double)delta);
        }
        else if (kind_ == K_GRADHELMHOLTZ || kind_ == K_DOUBLELAYER)
        {
            const double delta = std::max(std::abs(ki_) * H / 4., 1.0) *
                                 std::exp(-0.2 * (3.0 / std::sqrt(3.0)) * H * kr_);
            c = (int64_t)(int)std::ceil(delta);
        }
        else
        {
            const double delta = std::max(kr_ * H / 4., 1.);
            c = (int64_t)(int)std::ceil(delta);
        }
        out[i] = std::max<int64_t>(base[i] * c, 1);
    }
}

// cutoff_limit (ifgfoperator.hpp:1914, grad_helmholtz_ifgf.hpp:294-304)
double Operator::cutoff_limit(double H) const
{
    if (kind_ == K_GRADHELMHOLTZ && tol_ > 0)
        return std::max(1e-4, std::abs(kr_) * H / std::abs(std::log(tol_)));
    return 1e-4;
}

void Operator::orders(int step, int* o) const { order_for_box(step, o); }

void Operator::init(const double* srcs, int64_t ns, const double* tgts, int64_t nt,
                    const double* normals, const std::function<bool(double)>& cutoff,
                    bool plan_only)
{
    initialized_ = planned_ = false;
    const auto t0 = std::chrono::steady_clock::now();
    if (ns < 1 || nt < 1)
        throw Error(ERR_INVALID, "need at least one source and one target");
    if (!srcs || !tgts)
        throw Error(ERR_INVALID, "null point array");
    for (int64_t i = 0; i < 3 * ns; i++)
        if (!std::isfinite(srcs[i]))
            throw Error(ERR_INVALID, "non-finite source coordinate");
    for (int64_t i = 0; i < 3 * nt; i++)
        if (!std::isfinite(tgts[i]))
            throw Error(ERR_INVALID, "non-finite target coordinate");
    const bool need_n = kind_ == K_DOUBLELAYER || kind_ == K_COMBINEDFIELD;
    if (need_n && !normals && !plan_only)
        throw Error(ERR_INVALID, "this kernel needs source normals");
    if (need_n && normals)
        for (int64_t i = 0; i < 3 * ns; i++)
            if (!std::isfinite(normals[i]))
                throw Error(ERR_INVALID, "non-finite normal");
    // radial order reset of ifgfoperator.hpp:90 (fixed-order path), taken from
    // the constructor's order so that a repeated init does not compound it
    base_order_[0] = std::max(order0_ - 3, 2);
    order_for_box(0, lo_);
    order_for_box(1, hi_);
    for (int i = 0; i < 3; i++)
        if (lo_[i] < 1 || hi_[i] < 1)
            throw Error(ERR_INVALID, "interpolation order too low for this kernel (the low-order "
                                     "grid would have order < 1; use order >= 7)");
    if (lo_[0] * lo_[1] * lo_[2] > 4096 || hi_[0] * hi_[1] * hi_[2] > 2048 || lo_[0] > 16 ||
        lo_[1] > 16 || lo_[2] > 16)
        throw Error(ERR_INVALID, "interpolation order too high");

    plan_ = Plan();
    plan_.src.build(srcs, ns, leaf_);
    plan_.tgt.build(tgts, nt, leaf_);
    plan_.build_lists(cutoff);
    plan_.build_target_lists();

    const int L = plan_.src.num_levels();
    if (L > MAX_LEVELS)
        throw Error(ERR_INVALID, "octree deeper than supported");
    lv_.assign(L, LevelGeom());
    int64_t fmap_total = 0;
    for (int l = 0; l < L; l++)
    {
        LevelGeom& G = lv_[l];
        const TreeLevel& TL = plan_.src.levels[l];
        G.H = TL.side;
        const double smax = std::sqrt(3.0) / 3;
        double smin = cutoff_limit(G.H);
        if (smin >= smax)
            smin = smax - 0.05;
        G.dmin[0] = smin;
        G.dmax[0] = smax;
        G.dmin[1] = 0;
        G.dmax[1] = M_PI;
        G.dmin[2] = -M_PI;
        G.dmax[2] = M_PI;
        int64_t nf[3], nc[3];
        elements_for_box(G.H, 0, nf);
        elements_for_box(G.H, 1, nc);
        for (int d = 0; d < 3; d++)
        {
            if (nf[d] % nc[d] != 0)
                throw Error(ERR_INVALID, "fine grid is not a refinement of the coarse grid");
            G.nf[d] = (int)nf[d];
            G.nc[d] = (int)nc[d];
            G.hf[d] = (G.dmax[d] - G.dmin[d]) / (double)nf[d];
            G.hc[d] = (G.dmax[d] - G.dmin[d]) / (double)nc[d];
        }
        if (l == 0)
            for (int d = 0; d < 3; d++)
                fct_[d] = G.nf[d] / G.nc[d];
        for (int d = 0; d < 3; d++)
            if (G.nf[d] / G.nc[d] != fct_[d])
                throw Error(ERR_INVALID, "refinement factor differs between levels");
        G.nbox = (int)TL.size();
        G.box_off = (int)plan_.src.level_off[l];
        G.fmap_off = fmap_total;
        const int64_t nfe = nf[0] * nf[1] * nf[2];
        if (nfe > (1ll << 30))
            throw Error(ERR_INVALID, "cone grid too large");
        fmap_total += (int64_t)G.nbox * nfe;
    }
    if (fmap_total > (1ll << 34))
        throw Error(ERR_OOM, "dense cone maps would exceed 64 GB");
    planned_ = true;
    if (plan_only)
        return;
    setup_device(normals);
    initialized_ = true;
    init_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void Operator::setup_device(const double* normals)
{
    DeviceState& D = *dev_;
    const Tree& S = plan_.src;
    const Tree& Tt = plan_.tgt;
    const int L = S.num_levels();
    // source boxes, flattened by global id
    const int64_t nb = S.num_boxes_total();
    std::vector<double> bc(3 * nb), bH(nb);
    std::vector<int> bf(nb), bl(nb), bch(8 * nb), blev(nb);
    std::vector<unsigned char> bleaf(nb);
    for (int l = 0; l < L; l++)
    {
        const TreeLevel& TL = S.levels[l];
        const int64_t off = S.level_off[l];
        const int64_t coff = l + 1 < L ? S.level_off[l + 1] : 0;
        for (size_t b = 0; b < TL.size(); b++)
        {
            const int64_t g = off + (int64_t)b;
            for (int d = 0; d < 3; d++)
                bc[3 * g + d] = TL.center[3 * b + d];
            bH[g] = TL.sides[b];
            bf[g] = (int)TL.first[b];
            bl[g] = (int)TL.last[b];
            blev[g] = l;
            bleaf[g] = TL.leaf[b];
            for (int j = 0; j < 8; j++)
                bch[8 * g + j] = TL.child[8 * b + j] < 0 ? -1 : (int)(coff + TL.child[8 * b + j]);
        }
    }
    D.box_c.upload(bc);
    D.box_H.upload(bH);
    D.box_first.upload(bf);
    D.box_last.upload(bl);
    D.box_child.upload(bch);
    D.box_level.upload(blev);
    D.box_leaf.upload(bleaf);
    // points, SoA
    auto soa = [](const std::vector<double>& aos, int d) {
        std::vector<double> v(aos.size() / 3);
        for (size_t i = 0; i < v.size(); i++)
            v[i] = aos[3 * i + d];
        return v;
    };
    D.sx.upload(soa(S.pts, 0));
    D.sy.upload(soa(S.pts, 1));
    D.sz.upload(soa(S.pts, 2));
    D.tx.upload(soa(Tt.pts, 0));
    D.ty.upload(soa(Tt.pts, 1));
    D.tz.upload(soa(Tt.pts, 2));
    if (normals)
    {
        std::vector<double> n(3 * S.n);
        for (int64_t i = 0; i < S.n; i++) // onOctreeReady (double_layer_helmholtz_ifgf.hpp:29-35)
            for (int d = 0; d < 3; d++)
                n[3 * i + d] = normals[3 * S.perm[i] + d];
        D.nx.upload(soa(n, 0));
        D.ny.upload(soa(n, 1));
        D.nz.upload(soa(n, 2));
    }
    {
        std::vector<long long> sp(S.perm.begin(), S.perm.end()), tp(Tt.perm.begin(), Tt.perm.end());
        D.src_perm.upload(sp);
        D.tgt_perm.upload(tp);
    }
    // Chebyshev node local coordinates of the high-order (coarse) grid
    const int P_hi = hi_[0] * hi_[1] * hi_[2];
    const int P_lo = lo_[0] * lo_[1] * lo_[2];
    {
        auto r = cheb_nodes(hi_[0]), t = cheb_nodes(hi_[1]), p = cheb_nodes(hi_[2]);
        std::vector<double> nodes(3 * P_hi);
        for (int i = 0; i < hi_[2]; i++) // chebinterp.hpp:101-112
            for (int j = 0; j < hi_[1]; j++)
                for (int k = 0; k < hi_[0]; k++)
                {
                    const int id = i * hi_[1] * hi_[0] + j * hi_[0] + k;
                    nodes[3 * id] = r[k];
                    nodes[3 * id + 1] = t[j];
                    nodes[3 * id + 2] = p[i];
                }
        D.hi_nodes.upload(nodes);
        std::vector<double> A;
        for (int d = 0; d < 3; d++)
        {
            auto m = c2f_matrix(hi_[d], lo_[d], fct_[d]);
            A.insert(A.end(), m.begin(), m.end());
        }
        D.A.upload(A);
    }
    // target leaves
    {
        const int64_t ntl = (int64_t)plan_.tleaf_gid.size();
        std::vector<int> f(ntl), l(ntl);
        for (int64_t i = 0; i < ntl; i++)
        {
            int64_t g = plan_.tleaf_gid[i];
            int lev = (int)(std::upper_bound(Tt.level_off.begin(), Tt.level_off.end(), g) -
                            Tt.level_off.begin()) - 1;
            int64_t b = g - Tt.level_off[lev];
            f[i] = (int)Tt.levels[lev].first[b];
            l[i] = (int)Tt.levels[lev].last[b];
        }
        D.tl_first.upload(f);
        D.tl_last.upload(l);
        std::vector<long long> fo(plan_.tleaf_far_off.begin(), plan_.tleaf_far_off.end());
        std::vector<long long> no(plan_.tleaf_near_off.begin(), plan_.tleaf_near_off.end());
        D.tl_far_off.upload(fo);
        D.tl_near_off.upload(no);
        D.tl_far_src.upload(plan_.tleaf_far_src);
        D.tl_near_src.upload(plan_.tleaf_near_src);
        D.n_tleaf = (int)ntl;
    }

    // ---- active cones (octree.hpp:351-816) on the GPU ----
    int64_t fmap_total = 0;
    for (auto& G : lv_)
        fmap_total += (int64_t)G.nbox * G.nf[0] * G.nf[1] * G.nf[2];
    D.fmap.alloc(fmap_total);
    D.fmap.zero();
    int64_t cmax = 0, fmax_lvl = 0;
    for (auto& G : lv_)
    {
        cmax = std::max<int64_t>(cmax, (int64_t)G.nbox * G.nc[0] * G.nc[1] * G.nc[2]);
        fmax_lvl = std::max<int64_t>(fmax_lvl, (int64_t)G.nbox * G.nf[0] * G.nf[1] * G.nf[2]);
    }
    DevBuf<int> cmark, scan;
    cmark.alloc(cmax);
    scan.alloc(std::max(cmax, fmax_lvl));
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (int*)nullptr, (int*)nullptr,
                                  (int)std::max(cmax, fmax_lvl));
    DevBuf<unsigned char> tmp;
    tmp.alloc(std::max<size_t>(tmp_bytes, 1));
    TreeArgs TA{D.box_c.p, D.box_H.p, D.box_first.p, D.box_last.p, D.box_child.p, D.box_level.p,
                D.box_leaf.p};
    D.cc_box.clear();
    D.cc_el.clear();
    D.fc_box.clear();
    D.fc_el.clear();
    D.cc_box.resize(L);
    D.cc_el.resize(L);
    D.fc_box.resize(L);
    D.fc_el.resize(L);
    int64_t coarse_tot = 0, fine_tot = 0;
    leaf_evals_ = upward_evals_ = 0;
    for (int l = 0; l < L; l++)
    {
        LevelGeom& G = lv_[l];
        const int64_t nce = (int64_t)G.nc[0] * G.nc[1] * G.nc[2];
        const int64_t nfe = (int64_t)G.nf[0] * G.nf[1] * G.nf[2];
        const int64_t ncm = (int64_t)G.nbox * nce, nfm = (int64_t)G.nbox * nfe;
        IFGF_CUDA(cudaMemset(cmark.p, 0, ncm * sizeof(int)));
        // far pairs of this level
        std::vector<int> fs, f0, f1;
        for (int b = 0; b < G.nbox; b++)
        {
            const int64_t g = G.box_off + b;
            for (int64_t t : plan_.far[g])
            {
                int lev = (int)(std::upper_bound(Tt.level_off.begin(), Tt.level_off.end(), t) -
                                Tt.level_off.begin()) - 1;
                int64_t tb = t - Tt.level_off[lev];
                fs.push_back((int)g);
                f0.push_back((int)Tt.levels[lev].first[tb]);
                f1.push_back((int)Tt.levels[lev].last[tb]);
            }
        }
        if (!fs.empty())
        {
            DevBuf<int> dfs, df0, df1;
            dfs.upload(fs);
            df0.upload(f0);
            df1.upload(f1);
            mark_far_kernel<<<(unsigned)fs.size(), 128>>>(G, TA, dfs.p, df0.p, df1.p, D.tx.p,
                                                           D.ty.p, D.tz.p, D.fmap.p, cmark.p);
            IFGF_CUDA(cudaGetLastError());
            IFGF_CUDA(cudaDeviceSynchronize());
        }
        if (l > 0 && lv_[l - 1].n_coarse > 0)
        {
            mark_parent_kernel<<<(unsigned)lv_[l - 1].n_coarse, 128>>>(
                lv_[l - 1], G, TA, D.cc_box[l - 1].p, D.cc_el[l - 1].p, D.hi_nodes.p, P_hi,
                D.fmap.p, cmark.p);
            IFGF_CUDA(cudaGetLastError());
            IFGF_CUDA(cudaDeviceSynchronize());
        }
        // compaction
        auto compact = [&](int* map, int64_t n, int64_t n_el, int gbase, DevBuf<int>& lbox,
                           DevBuf<int>& lel) -> int64_t {
            if (n == 0)
                return 0;
            size_t tb = tmp.n;
            IFGF_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, map, scan.p, (int)n));
            int last_scan = 0, last_mark = 0;
            IFGF_CUDA(cudaMemcpy(&last_scan, scan.p + n - 1, sizeof(int), cudaMemcpyDeviceToHost));
            IFGF_CUDA(cudaMemcpy(&last_mark, map + n - 1, sizeof(int), cudaMemcpyDeviceToHost));
            const int64_t cnt = (int64_t)last_scan + (last_mark ? 1 : 0);
            lbox.alloc(std::max<int64_t>(cnt, 1));
            lel.alloc(std::max<int64_t>(cnt, 1));
            const int thr = 256;
            const int blocks = (int)std::min<int64_t>((n + thr - 1) / thr, 148 * 32);
            finalize_map_kernel<<<blocks, thr>>>(map, scan.p, n, (int)n_el, G.box_off, gbase,
                                                 lbox.p, lel.p);
            IFGF_CUDA(cudaGetLastError());
            IFGF_CUDA(cudaDeviceSynchronize());
            return cnt;
        };
        G.n_coarse = compact(cmark.p, ncm, nce, 0, D.cc_box[l], D.cc_el[l]);
        G.coarse_off = coarse_tot;
        coarse_tot += G.n_coarse;
        G.n_fine = compact(D.fmap.p + G.fmap_off, nfm, nfe, (int)fine_tot, D.fc_box[l], D.fc_el[l]);
        G.fine_off = fine_tot;
        fine_tot += G.n_fine;
        if (fine_tot > (1ll << 31) - 1)
            throw Error(ERR_OOM, "too many active fine cones");
        // work counts of the flop model
        if (G.n_coarse > 0)
        {
            std::vector<int> cb(G.n_coarse);
            IFGF_CUDA(cudaMemcpy(cb.data(), D.cc_box[l].p, cb.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost));
            for (int g : cb)
            {
                if (bleaf[g])
                    leaf_evals_ += (double)P_hi * (bl[g] - bf[g]);
                else
                {
                    int nch = 0;
                    for (int j = 0; j < 8; j++)
                        nch += bch[8 * g + j] >= 0;
                    upward_evals_ += (double)P_hi * nch;
                }
            }
        }
    }
    n_coarse_total_ = coarse_tot;
    n_fine_total_ = fine_tot;
    D.lv.upload(lv_);
    int64_t cmax_active = 0;
    for (auto& G : lv_)
        cmax_active = std::max<int64_t>(cmax_active, G.n_coarse);
    D.cvals.alloc((size_t)std::max<int64_t>(cmax_active, 1) * P_hi);
    D.fcoef.alloc((size_t)std::max<int64_t>(fine_tot, 1) * P_lo);
    D.fcoef.zero(); // fine cones without an active coarse parent stay zero
    D.w.alloc(S.n);
    D.err.alloc(1);
    D.err.zero();
    // launch shapes
    const int npt = (P_hi + 511) / 512;
    D.cv_threads = ((P_hi + npt - 1) / npt + 31) / 32 * 32;
    if (npt > CV_MAXNPT)
        throw Error(ERR_INVALID, "interpolation order too high");
    const int F0 = fct_[0] * lo_[0], F1 = fct_[1] * lo_[1];
    const size_t sz2 = std::max<size_t>((size_t)F0 * hi_[1] * hi_[2], (size_t)F0 * F1 * lo_[2]);
    D.c2f_smem = (P_hi + sz2 + (size_t)F0 * F1 * hi_[2]) * sizeof(double2);
    if (D.c2f_smem > 220 * 1024)
        throw Error(ERR_INVALID, "interpolation order too high for the coarse-to-fine kernel");
    IFGF_CUDA(cudaFuncSetAttribute(coarse_to_fine_kernel,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D.c2f_smem));
}

// FP64 direct sum at selected targets: one CTA per target, Kahan-compensated
// per-thread partial sums, then a pairwise block reduction.
template <int KIND>
__global__ void __launch_bounds__(256) direct_eval_kernel(SrcArgs S, const double2* __restrict__ w,
                                                          int ns, const double* __restrict__ tx,
                                                          const double* __restrict__ ty,
                                                          const double* __restrict__ tz,
                                                          const int* __restrict__ tpos,
                                                          KParams kp, double2* out)
{
    using P = Plugin<KIND>;
    __shared__ double sr[256], si[256];
    const int j = tpos[blockIdx.x];
    const double y0 = tx[j], y1 = ty[j], y2 = tz[j];
    double ar = 0, ai = 0, cr = 0, ci = 0;
    for (int s = threadIdx.x; s < ns; s += blockDim.x)
    {
        const double x[3] = {S.sx[s] - y0, S.sy[s] - y1, S.sz[s] - y2};
        const double nv[3] = {P::needs_normals ? S.nx[s] : 0.0, P::needs_normals ? S.ny[s] : 0.0,
                              P::needs_normals ? S.nz[s] : 0.0};
        const cplx<double> g = P::kernel(x, nv, kp);
        const double2 wv = w[s];
        const double vr = wv.x * g.re - wv.y * g.im, vi = wv.x * g.im + wv.y * g.re;
        double yr = vr - cr, tr = ar + yr;
        cr = (tr - ar) - yr;
        ar = tr;
        double yi = vi - ci, ti = ai + yi;
        ci = (ti - ai) - yi;
        ai = ti;
    }
    sr[threadIdx.x] = ar;
    si[threadIdx.x] = ai;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1)
    {
        if (threadIdx.x < h)
        {
            sr[threadIdx.x] += sr[threadIdx.x + h];
            si[threadIdx.x] += si[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        out[blockIdx.x] = make_double2(sr[0], si[0]);
}

enum ProfClass
{
    PROF_PERMUTE = 0,
    PROF_COARSE = 1,
    PROF_C2F = 2,
    PROF_EVAL = 3
};

// Records CUDA events around every launch when profiling is on.
struct LaunchLog
{
    DeviceState& D;
    cudaStream_t st;
    bool on;
    std::vector<int> cls;
    int n = 0;
    void begin(int c)
    {
        if (!on)
            return;
        ensure(n + 1);
        cls.push_back(c);
        IFGF_CUDA(cudaEventRecord(D.prof_ev[2 * n], st));
    }
    void end()
    {
        if (!on)
            return;
        IFGF_CUDA(cudaEventRecord(D.prof_ev[2 * n + 1], st));
        n++;
    }
    void ensure(int m)
    {
        while ((int)D.prof_ev.size() < 2 * m)
        {
            cudaEvent_t e;
            IFGF_CUDA(cudaEventCreate(&e));
            D.prof_ev.push_back(e);
        }
    }
};

template <int KIND>
static int launch_kernels(DeviceState& D, const std::vector<LevelGeom>& lv, const int* lo,
                          const int* hi, const int* fct, const KParams& kp, bool real,
                          const void* d_w, void* d_u, cudaStream_t st, LaunchLog& log)
{
    const int L = (int)lv.size();
    const int P_hi = hi[0] * hi[1] * hi[2];
    const int P_lo = lo[0] * lo[1] * lo[2];
    const int64_t ns = (int64_t)D.w.n;
    int launches = 0;
    TreeArgs TA{D.box_c.p, D.box_H.p, D.box_first.p, D.box_last.p, D.box_child.p, D.box_level.p,
                D.box_leaf.p};
    SrcArgs SA{D.sx.p, D.sy.p, D.sz.p, D.nx.p, D.ny.p, D.nz.p};
    {
        const int thr = 256;
        const int blocks = (int)std::min<int64_t>((ns + thr - 1) / thr, 148 * 16);
        log.begin(PROF_PERMUTE);
        permute_weights_kernel<<<blocks, thr, 0, st>>>((const double*)d_w, real ? 1 : 0,
                                                       D.src_perm.p, D.w.p, ns);
        IFGF_CUDA(cudaGetLastError());
        log.end();
        launches++;
    }
    for (int l = L - 1; l >= 0; l--)
    {
        const LevelGeom& G = lv[l];
        if (G.n_coarse == 0)
            continue;
        CoarseArgs ca;
        ca.G = G;
        ca.GC = l + 1 < L ? lv[l + 1] : G;
        ca.T = TA;
        ca.S = SA;
        ca.cc_box = D.cc_box[l].p;
        ca.cc_el = D.cc_el[l].p;
        ca.hi_nodes = D.hi_nodes.p;
        ca.w = D.w.p;
        ca.fmap = D.fmap.p;
        ca.fcoef = D.fcoef.p;
        ca.cvals = D.cvals.p;
        ca.err = D.err.p;
        ca.P_hi = P_hi;
        ca.P_lo = P_lo;
        for (int d = 0; d < 3; d++)
            ca.lo[d] = lo[d];
        ca.kp = kp;
        const int thr = D.cv_threads;
        const size_t smem = (size_t)8 * thr * sizeof(double);
        log.begin(PROF_COARSE);
        coarse_values_kernel<KIND><<<(unsigned)G.n_coarse, thr, smem, st>>>(ca);
        IFGF_CUDA(cudaGetLastError());
        log.end();
        C2FArgs fa;
        fa.G = G;
        fa.cc_box = D.cc_box[l].p;
        fa.cc_el = D.cc_el[l].p;
        fa.cvals = D.cvals.p;
        fa.A = D.A.p;
        fa.fmap = D.fmap.p;
        fa.fcoef = D.fcoef.p;
        for (int d = 0; d < 3; d++)
        {
            fa.hi[d] = hi[d];
            fa.lo[d] = lo[d];
            fa.f[d] = fct[d];
        }
        fa.P_hi = P_hi;
        fa.P_lo = P_lo;
        log.begin(PROF_C2F);
        coarse_to_fine_kernel<<<(unsigned)G.n_coarse, 256, D.c2f_smem, st>>>(fa);
        IFGF_CUDA(cudaGetLastError());
        log.end();
        launches += 2;
    }
    EvalArgs ea;
    ea.lv = D.lv.p;
    ea.T = TA;
    ea.S = SA;
    ea.tx = D.tx.p;
    ea.ty = D.ty.p;
    ea.tz = D.tz.p;
    ea.tgt_perm = D.tgt_perm.p;
    ea.tl_first = D.tl_first.p;
    ea.tl_last = D.tl_last.p;
    ea.far_off = D.tl_far_off.p;
    ea.far_src = D.tl_far_src.p;
    ea.near_off = D.tl_near_off.p;
    ea.near_src = D.tl_near_src.p;
    ea.w = D.w.p;
    ea.fmap = D.fmap.p;
    ea.fcoef = D.fcoef.p;
    ea.out = (double*)d_u;
    ea.real_out = real ? 1 : 0;
    ea.err = D.err.p;
    ea.P_lo = P_lo;
    for (int d = 0; d < 3; d++)
        ea.lo[d] = lo[d];
    ea.kp = kp;
    if (D.n_tleaf > 0)
    {
        log.begin(PROF_EVAL);
        target_eval_kernel<KIND><<<D.n_tleaf, EVAL_THREADS, 0, st>>>(ea);
        IFGF_CUDA(cudaGetLastError());
        log.end();
        launches++;
    }
    return launches;
}

template <int KIND>
static void launch_direct(DeviceState& D, const KParams& kp, const int* d_tpos, int nt,
                          double2* d_out)
{
    SrcArgs SA{D.sx.p, D.sy.p, D.sz.p, D.nx.p, D.ny.p, D.nz.p};
    direct_eval_kernel<KIND><<<nt, 256>>>(SA, D.w.p, (int)D.w.n, D.tx.p, D.ty.p, D.tz.p, d_tpos,
                                          kp, d_out);
    IFGF_CUDA(cudaGetLastError());
}

#define IFGF_DISPATCH(KINDVAR, CALL)                                                          \
    switch (KINDVAR)                                                                           \
    {                                                                                          \
    case K_LAPLACE: { constexpr int KK = K_LAPLACE; CALL; } break;                            \
    case K_HELMHOLTZ: { constexpr int KK = K_HELMHOLTZ; CALL; } break;                        \
    case K_MODHELMHOLTZ: { constexpr int KK = K_MODHELMHOLTZ; CALL; } break;                  \
    case K_GRADHELMHOLTZ: { constexpr int KK = K_GRADHELMHOLTZ; CALL; } break;                \
    case K_DOUBLELAYER: { constexpr int KK = K_DOUBLELAYER; CALL; } break;                    \
    case K_COMBINEDFIELD: { constexpr int KK = K_COMBINEDFIELD; CALL; } break;                \
    }

void Operator::launch_mult(const void* d_w, void* d_u, void* stream, bool timed)
{
    if (!initialized_)
        throw Error(ERR_STATE, "mult called before init");
    if (!d_w || !d_u)
        throw Error(ERR_INVALID, "null density or result buffer");
    const KParams kp{kr_, ki_, dx_};
    cudaStream_t st = (cudaStream_t)stream;
    DeviceState& D = *dev_;
    LaunchLog log{D, st, profiling_ || timed};
    int launches = 0;
    IFGF_DISPATCH(kind_, launches = launch_kernels<KK>(D, lv_, lo_, hi_, fct_, kp, is_real(), d_w,
                                                        d_u, st, log));
    launches_per_mult_ = launches;
    if (log.on && log.n > 0)
    {
        IFGF_CUDA(cudaEventSynchronize(D.prof_ev[2 * log.n - 1]));
        double cls_ms[NPROF] = {0, 0, 0, 0};
        for (int i = 0; i < log.n; i++)
        {
            float ms = 0;
            IFGF_CUDA(cudaEventElapsedTime(&ms, D.prof_ev[2 * i], D.prof_ev[2 * i + 1]));
            cls_ms[log.cls[i]] += ms;
            if (profiling_)
            {
                prof_ms_[log.cls[i]] += ms;
                prof_launches_[log.cls[i]]++;
            }
        }
        float tot = 0;
        IFGF_CUDA(cudaEventElapsedTime(&tot, D.prof_ev[0], D.prof_ev[2 * log.n - 1]));
        if (profiling_)
            mults_profiled_++;
        last_.permute = cls_ms[PROF_PERMUTE];
        last_.coarse = cls_ms[PROF_COARSE];
        last_.c2f = cls_ms[PROF_C2F];
        last_.eval = cls_ms[PROF_EVAL];
        last_.total = tot;
    }
}

void Operator::set_profiling(bool on)
{
    profiling_ = on;
    for (int i = 0; i < NPROF; i++)
    {
        prof_launches_[i] = 0;
        prof_ms_[i] = 0;
    }
    mults_profiled_ = 0;
}

void Operator::mult_device(const void* d_w, void* d_u, void* stream)
{
    launch_mult(d_w, d_u, stream, false);
}

void Operator::mult_host(const void* w, void* u, int64_t batch)
{
    if (!initialized_)
        throw Error(ERR_STATE, "mult called before init");
    if (!w || !u)
        throw Error(ERR_INVALID, "null density or result buffer");
    if (batch < 1)
        throw Error(ERR_INVALID, "batch must be >= 1");
    DeviceState& D = *dev_;
    const size_t per = is_real() ? 1 : 2;
    const size_t nw = per * (size_t)n_src(), nu = per * (size_t)n_tgt();
    if (D.io_w.n < nw)
        D.io_w.alloc(nw);
    if (D.io_u.n < nu)
        D.io_u.alloc(nu);
    for (int64_t b = 0; b < batch; b++)
    {
        IFGF_CUDA(cudaMemcpy(D.io_w.p, (const double*)w + b * nw, nw * sizeof(double),
                             cudaMemcpyHostToDevice));
        launch_mult(D.io_w.p, D.io_u.p, nullptr, true);
        IFGF_CUDA(cudaMemcpy((double*)u + b * nu, D.io_u.p, nu * sizeof(double),
                             cudaMemcpyDeviceToHost));
    }
    IFGF_CUDA(cudaMemcpy(&missing_, D.err.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
}

void Operator::mult_device_external_scratch(const void* d_w, void* d_u, void* stream,
                                            void* scratch, size_t scratch_bytes)
{
    if (!initialized_)
        throw Error(ERR_STATE, "mult called before init");
    if (!d_w || !d_u || !scratch)
        throw Error(ERR_INVALID, "null density, result or scratch buffer");
    DeviceState& D = *dev_;
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t bw = up(D.w.n * sizeof(double2)), bc = up(D.cvals.n * sizeof(double2)),
                 bf = up(D.fcoef.n * sizeof(double2));
    const size_t need = bw + bc + bf;
    if (need > scratch_bytes)
        throw Error(ERR_INVALID, "this operator needs " + std::to_string(need) +
                                     " bytes of matvec scratch; the fixed no-allocation scratch "
                                     "holds " + std::to_string(scratch_bytes) +
                                     " bytes (use ifgf_mult_device for larger problems)");
    unsigned char* base = static_cast<unsigned char*>(scratch);
    double2* w = reinterpret_cast<double2*>(base);
    double2* cv = reinterpret_cast<double2*>(base + bw);
    double2* fc = reinterpret_cast<double2*>(base + bw + bc);
    cudaStream_t st = (cudaStream_t)stream;
    // fine cones without an active coarse parent must read as zero; the
    // shared scratch still holds the previous call's coefficients
    IFGF_CUDA(cudaMemsetAsync(fc, 0, D.fcoef.n * sizeof(double2), st));
    // point the operator's scratch buffers at the caller's region for this
    // call only (sizes unchanged), restoring them on every exit path
    struct Redirect
    {
        DeviceState& D;
        double2 *w, *cv, *fc;
        ~Redirect()
        {
            D.w.p = w;
            D.cvals.p = cv;
            D.fcoef.p = fc;
        }
    } restore{D, D.w.p, D.cvals.p, D.fcoef.p};
    D.w.p = w;
    D.cvals.p = cv;
    D.fcoef.p = fc;
    const KParams kp{kr_, ki_, dx_};
    LaunchLog log{D, st, false}; // no events: this path creates no resources
    IFGF_DISPATCH(kind_, launch_kernels<KK>(D, lv_, lo_, hi_, fct_, kp, is_real(), d_w, d_u, st, log));
}

void Operator::direct_eval(const void* w, const int64_t* tidx, int64_t nt, void* out)
{
    if (!initialized_)
        throw Error(ERR_STATE, "direct_eval called before init");
    if (!w || !out || (nt > 0 && !tidx))
        throw Error(ERR_INVALID, "null buffer");
    if (nt <= 0)
        return;
    DeviceState& D = *dev_;
    // sorted position of each requested original target index
    const auto& perm = plan_.tgt.perm;
    std::vector<int64_t> inv(perm.size());
    for (size_t i = 0; i < perm.size(); i++)
        inv[perm[i]] = (int64_t)i;
    std::vector<int> pos(nt);
    for (int64_t q = 0; q < nt; q++)
    {
        if (tidx[q] < 0 || tidx[q] >= (int64_t)perm.size())
            throw Error(ERR_INVALID, "target index out of range");
        pos[q] = (int)inv[tidx[q]];
    }
    const size_t per = is_real() ? 1 : 2;
    const size_t nw = per * (size_t)n_src();
    if (D.io_w.n < nw)
        D.io_w.alloc(nw);
    IFGF_CUDA(cudaMemcpy(D.io_w.p, w, nw * sizeof(double), cudaMemcpyHostToDevice));
    {
        const int64_t ns = (int64_t)D.w.n;
        const int thr = 256;
        const int blocks = (int)std::min<int64_t>((ns + thr - 1) / thr, 148 * 16);
        permute_weights_kernel<<<blocks, thr>>>(D.io_w.p, is_real() ? 1 : 0, D.src_perm.p, D.w.p, ns);
        IFGF_CUDA(cudaGetLastError());
    }
    DevBuf<int> dpos;
    dpos.upload(pos);
    DevBuf<double2> dout;
    dout.alloc(nt);
    const KParams kp{kr_, ki_, dx_};
    IFGF_DISPATCH(kind_, launch_direct<KK>(D, kp, dpos.p, (int)nt, dout.p));
    std::vector<double2> h(nt);
    IFGF_CUDA(cudaMemcpy(h.data(), dout.p, nt * sizeof(double2), cudaMemcpyDeviceToHost));
    double* o = (double*)out;
    for (int64_t q = 0; q < nt; q++)
    {
        if (is_real())
            o[q] = h[q].x;
        else
        {
            o[2 * q] = h[q].x;
            o[2 * q + 1] = h[q].y;
        }
    }
}


void Operator::level_grid(int level, int step, int64_t* n) const
{
    if (level < 0 || level >= (int)lv_.size())
        throw Error(ERR_INVALID, "level out of range");
    for (int d = 0; d < 3; d++)
        n[d] = step == 0 ? lv_[level].nf[d] : lv_[level].nc[d];
}

std::vector<int64_t> Operator::box_cones(int level, int64_t box, int step) const
{
    if (level < 0 || level >= (int)lv_.size())
        throw Error(ERR_INVALID, "level out of range");
    const LevelGeom& G = lv_[level];
    if (box < 0 || box >= G.nbox)
        throw Error(ERR_INVALID, "box out of range");
    const int64_t cnt = step == 0 ? G.n_fine : G.n_coarse;
    std::vector<int64_t> out;
    if (cnt == 0)
        return out;
    std::vector<int> b(cnt), e(cnt);
    const DeviceState& D = *dev_;
    const auto& lb = step == 0 ? D.fc_box[level] : D.cc_box[level];
    const auto& le = step == 0 ? D.fc_el[level] : D.cc_el[level];
    IFGF_CUDA(cudaMemcpy(b.data(), lb.p, cnt * sizeof(int), cudaMemcpyDeviceToHost));
    IFGF_CUDA(cudaMemcpy(e.data(), le.p, cnt * sizeof(int), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < cnt; i++)
        if (b[i] == G.box_off + box)
            out.push_back(e[i]);
    return out;
}

std::string Operator::stats_json() const
{
    std::ostringstream o;
    o.precision(10);
    o << "{\"kind\":" << kind_ << ",\"precision\":" << precision_ << ",\"n_src\":" << n_src()
      << ",\"n_tgt\":" << n_tgt() << ",\"order_high\":[" << hi_[0] << "," << hi_[1] << ","
      << hi_[2] << "],\"order_low\":[" << lo_[0] << "," << lo_[1] << "," << lo_[2] << "]"
      << ",\"levels\":" << lv_.size() << ",\"boxes\":[";
    for (size_t l = 0; l < lv_.size(); l++)
        o << (l ? "," : "") << lv_[l].nbox;
    o << "],\"coarse_grid\":[";
    for (size_t l = 0; l < lv_.size(); l++)
        o << (l ? "," : "") << "[" << lv_[l].nc[0] << "," << lv_[l].nc[1] << "," << lv_[l].nc[2] << "]";
    o << "],\"active_coarse\":[";
    for (size_t l = 0; l < lv_.size(); l++)
        o << (l ? "," : "") << lv_[l].n_coarse;
    o << "],\"active_fine\":[";
    for (size_t l = 0; l < lv_.size(); l++)
        o << (l ? "," : "") << lv_[l].n_fine;
    o << "],\"near_pairs\":" << plan_.n_near_pairs << ",\"far_pairs\":" << plan_.n_far_pairs
      << ",\"dropped_pairs\":" << plan_.n_dropped
      << ",\"near_point_pairs\":" << plan_.near_point_pairs
      << ",\"far_target_evals\":" << plan_.far_target_evals
      << ",\"leaf_factor_evals\":" << leaf_evals_ << ",\"upward_node_evals\":" << upward_evals_
      << ",\"coarse_cones_total\":" << n_coarse_total_ << ",\"fine_cones_total\":" << n_fine_total_
      << ",\"target_leaves\":" << dev_->n_tleaf << ",\"missing_cone_lookups\":" << missing_
      << ",\"init_ms\":" << init_ms_ << ",\"launches_per_mult\":" << launches_per_mult_
      << ",\"last_mult_ms\":{\"permute\":" << last_.permute << ",\"coarse_values\":" << last_.coarse
      << ",\"coarse_to_fine\":" << last_.c2f << ",\"target_eval\":" << last_.eval
      << ",\"total\":" << last_.total << "},\"profile\":{\"mults\":" << mults_profiled_;
    const char* names[NPROF] = {"permute", "coarse_values", "coarse_to_fine", "target_eval"};
    for (int i = 0; i < NPROF; i++)
        o << ",\"" << names[i] << "\":{\"launches\":" << prof_launches_[i] << ",\"ms\":" << prof_ms_[i]
          << "}";
    o << "}}";
    return o.str();
}

} // namespace ifgf
