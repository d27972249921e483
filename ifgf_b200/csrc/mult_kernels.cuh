// Matvec kernels of the IFGF pipeline (IfgfOperator::mult,
// ifgfoperator.hpp:246-867), restructured level-synchronously for sm_100a:
//
//   permute_weights     w -> Morton order (ifgfoperator.hpp:252-254)
//   per level, deepest first:
//     leaf_sample       nodal values of leaf boxes' coarse cones
//                       (evaluateFactoredKernel at the cone's Chebyshev nodes,
//                       ifgfoperator.hpp:1057-1073, 423-462)
//     upward            nodal values of other boxes' coarse cones: children's
//                       fine interpolants at the nodes x transfer_factor
//                       (transferInterp, ifgfoperator.hpp:1639-1705, 633-688)
//     coarse_to_fine    chebtransform, coarseToFine and the fine chebtransform
//                       (ifgfoperator.hpp:1087-1124, 1539-1637) as three
//                       per-dimension matrix products
//   target_eval         per target leaf: near field + far field of every
//                       admissible source box, written in caller order
//                       (ifgfoperator.hpp:900-1012, 1707-1891, 862-866)
//
// Included by one translation unit per kernel plug-in (kernels_k<KIND>.cu).
#pragma once

#include <type_traits>

#include "mult.hpp"

namespace ifgf
{

// ---------------------------------------------------------------------------
// Tensor-product Chebyshev sums with compile-time orders (registers only);
// N0 = 0 selects the runtime-order fallback.
// ---------------------------------------------------------------------------
template <int N> __device__ __forceinline__ void cheb_T(double x, double* t)
{
    t[0] = 1.0;
    if (N > 1)
        t[1] = x;
    const double x2 = 2.0 * x;
#pragma unroll
    for (int i = 2; i < N; i++)
        t[i] = fma(x2, t[i - 1], -t[i - 2]);
}

template <int N0, int N1, int N2> struct Cheb
{
    __device__ static __forceinline__ cplx<double> eval(const double2* __restrict__ c,
                                                        const double* x, const int*)
    {
        double t0[N0], t1[N1], t2[N2];
        cheb_T<N0>(x[0], t0);
        cheb_T<N1>(x[1], t1);
        cheb_T<N2>(x[2], t2);
        double ar = 0, ai = 0;
#pragma unroll
        for (int k = 0; k < N2; k++)
        {
            double br = 0, bi = 0;
#pragma unroll
            for (int j = 0; j < N1; j++)
            {
                double cr = 0, ci = 0;
#pragma unroll
                for (int i = 0; i < N0; i++)
                {
                    const double2 v = __ldg(c + i + N0 * (j + N1 * k));
                    cr = fma(v.x, t0[i], cr);
                    ci = fma(v.y, t0[i], ci);
                }
                br = fma(cr, t1[j], br);
                bi = fma(ci, t1[j], bi);
            }
            ar = fma(br, t2[k], ar);
            ai = fma(bi, t2[k], ai);
        }
        return {ar, ai};
    }
};

template <> struct Cheb<0, 0, 0>
{
    __device__ static __forceinline__ cplx<double> eval(const double2* __restrict__ c,
                                                        const double* x, const int* n)
    {
        return cheb_eval3<16>(c, x, n);
    }
};

// ---------------------------------------------------------------------------
static __global__ void permute_weights_kernel(const double* __restrict__ in, int real_in,
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

constexpr int NPT = 2;           // coarse-cone nodes per thread
constexpr int NODE_THREADS = 256; // threads of the leaf / upward CTAs (max)

struct LeafArgs
{
    LevelGeom G;
    TreeArgs T;
    SrcArgs S;
    const int* __restrict__ cc_box;
    const int* __restrict__ cc_el;
    const int* __restrict__ idx;
    const double* __restrict__ hi_nodes;
    const double2* __restrict__ w;
    double2* cvals;
    int P_hi;
    KParams kp;
};

// Cartesian position of Chebyshev node n of coarse cone `el` of a box.
__device__ __forceinline__ void node_position(const LevelGeom& G, int el, int n,
                                              const double* __restrict__ hi_nodes,
                                              const double* xc, double H, double* y)
{
    const double loc[3] = {hi_nodes[3 * n], hi_nodes[3 * n + 1], hi_nodes[3 * n + 2]};
    double s[3];
    from_local(el, loc, G.dmin, G.hc, G.nc, s);
    interp_to_cart(s, xc, H, y);
}

// One CTA per coarse cone of a leaf box: sum over the leaf's sources
// (staged in shared memory) at NPT nodes per thread.
template <int KIND>
__global__ void __launch_bounds__(NODE_THREADS) leaf_sample_kernel(LeafArgs a)
{
    using P = Plugin<KIND>;
    extern __shared__ double sm[];
    const int c = a.idx[blockIdx.x];
    const int node0 = blockIdx.y * NPT * blockDim.x; // node chunk of this CTA
    const int box = a.cc_box[c], el = a.cc_el[c];
    const double xc[3] = {a.T.box_c[3 * box], a.T.box_c[3 * box + 1], a.T.box_c[3 * box + 2]};
    const double H = a.T.box_H[box];
    double y[NPT][3], dc[NPT];
    cplx<double> acc[NPT];
#pragma unroll
    for (int q = 0; q < NPT; q++)
    {
        const int n = node0 + threadIdx.x + q * blockDim.x;
        acc[q] = {0.0, 0.0};
        y[q][0] = y[q][1] = y[q][2] = 0;
        dc[q] = 0;
        if (n < a.P_hi)
        {
            node_position(a.G, el, n, a.hi_nodes, xc, H, y[q]);
            const double e0 = y[q][0] - xc[0], e1 = y[q][1] - xc[1], e2 = y[q][2] - xc[2];
            dc[q] = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
        }
    }
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
        for (int q = 0; q < NPT; q++)
        {
            if (node0 + threadIdx.x + q * blockDim.x >= a.P_hi)
                continue;
            for (int i = 0; i < cnt; i++)
            {
                const double av[3] = {xs[i] - y[q][0], ys[i] - y[q][1], zs[i] - y[q][2]};
                const double nv[3] = {P::needs_normals ? n0[i] : 0.0, P::needs_normals ? n1[i] : 0.0,
                                      P::needs_normals ? n2[i] : 0.0};
                acc[q] = cadd(acc[q], P::factored(av, nv, {wr[i], wi[i]}, y[q], dc[q], a.kp));
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NPT; q++)
    {
        const int n = node0 + threadIdx.x + q * blockDim.x;
        if (n < a.P_hi)
            a.cvals[(size_t)c * a.P_hi + n] = make_double2(acc[q].re, acc[q].im);
    }
}

struct UpArgs
{
    LevelGeom G;  // this (parent) level
    LevelGeom GC; // child level
    TreeArgs T;
    const int* __restrict__ cc_box;
    const int* __restrict__ cc_el;
    const int* __restrict__ idx;
    const int* __restrict__ slot;
    const UpGeo64* __restrict__ geo64;
    const UpGeo32* __restrict__ geo32;
    int P_pad;
    // [slot][octant][fe_pad + 1]: (element, first group) per run, then a
    // sentinel (-1, groups of the row)
    const int2* __restrict__ fe_list;
    int fe_pad;
    int rch; // runs staged at a time by the staged kernel
    // batched right-hand sides (staged kernel): blockIdx.y selects the plane
    long long cv_plane, fc_plane;
    const double* __restrict__ hi_nodes;
    const int* __restrict__ fmap;
    const double2* __restrict__ fcoef;
    double2* cvals;
    unsigned long long* err;
    int P_hi, P_lo;
    int lo[3];
    KParams kp;
    // staged kernel with MK: wavenumber of plane blockIdx.y, and geo32 holds
    // distance tables (tr = d - d_parent, ti = d_parent / d)
    const KParams* kp_plane = nullptr;
    // tensor-core kernel: row tiles (first up_idx position, cones, first
    // plane, planes) and the status word its bounded waits report into
    const int4* tc_tiles = nullptr;
    unsigned* tc_status = nullptr;
    // tensor-core kernel: the level's basis images (null: the kernel builds
    // the basis rows itself), with the byte offset of every (slot, octant)
    const unsigned char* tc_img = nullptr;
    const long long* tc_img_off = nullptr;
};

// One CTA per coarse cone of a box with children (CTAs ordered by cone
// element, so consecutive CTAs share their geometry-table rows in L2): every
// child's fine interpolant at the cone's nodes, times the centre-shift
// factor, with the box-independent geometry read from the level's table.
// Should a tabulated element be inactive in this child (the table works in
// coordinates relative to the parent, the activation in absolute ones), the
// node is recomputed from absolute coordinates as the reference does.
template <int KIND, int N0, int N1, int N2>
__device__ __forceinline__ bool upward_fallback64(const UpArgs& a, int box, int el, int n, int cb,
                                                  const int* fm, cplx<double>& v_out)
{
    using P = Plugin<KIND>;
    const LevelGeom& C = a.GC;
    const double xc[3] = {a.T.box_c[3 * box], a.T.box_c[3 * box + 1], a.T.box_c[3 * box + 2]};
    double y[3];
    node_position(a.G, el, n, a.hi_nodes, xc, a.T.box_H[box], y);
    const double p0 = y[0] - a.T.box_c[3 * cb], p1 = y[1] - a.T.box_c[3 * cb + 1],
                 p2 = y[2] - a.T.box_c[3 * cb + 2];
    double s[3], loc[3];
    cart_to_interp(p0, p1, p2, a.T.box_H[cb], s);
    const int fe = element_for_point(s, C.dmin, C.dmax, C.hfi, C.nf);
    if (fe < 0)
        return false;
    const int gf = fm[fe];
    if (gf < 0)
    {
        atomicAdd(a.err, 1ull);
        return false;
    }
    to_local(fe, s, C.dmin, C.hf, C.hfi, C.nf, loc);
    const cplx<double> v = Cheb<N0, N1, N2>::eval(a.fcoef + (size_t)gf * a.P_lo, loc, a.lo);
    const double e0 = y[0] - xc[0], e1 = y[1] - xc[1], e2 = y[2] - xc[2];
    v_out = cmul(v, P::transfer(p0 * p0 + p1 * p1 + p2 * p2, e0 * e0 + e1 * e1 + e2 * e2, a.kp));
    return true;
}

// Builds one level's upward geometry (FP64 values and their FP32 copies):
// the parent box is centred at the origin, child o at off[o].  One CTA per
// (slot, octant) row.  The row lists the nodes that fall inside the child's
// domain, sorted by child element, each element's run padded with skipped
// entries to a multiple of UPGEO_RUN so that a group of UPGEO_RUN entries
// always shares one element.  fill = 2 writes distance tables instead of
// centre-shift factors (UpGeo32 tr = d - d_parent, ti = d_parent / d; no
// UpGeo64 table).  fill = 0 only measures the row: its padded
// length and its number of element runs (row_len[2 row], row_len[2 row + 1]).
// fill = 1 also lists each row's distinct elements in run order
// with the group at which each run starts (fe_list[row (fe_pad + 1) + r] =
// (element, first group)), followed by a sentinel (-1, groups of the row),
// and stores the run index r of every entry in
// UpGeo32::pad, so that a kernel can stage one coefficient block per run.
constexpr int UPGEO_RUN = 4;

template <int KIND>
__global__ void __launch_bounds__(256) build_upgeo_kernel(LevelGeom PG, LevelGeom CG, double pH,
                                                          double cH, const double* __restrict__ off,
                                                          const int* __restrict__ slot_el,
                                                          const double* __restrict__ hi_nodes,
                                                          int P_hi, KParams kp, int fill, int P_pad,
                                                          int* row_len, UpGeo64* g64, UpGeo32* g32,
                                                          int fe_pad, int2* fe_list)
{
    using P = Plugin<KIND>;
    // key[P_hi] | sorted node[P_hi] | padded position[P_hi] | run index[P_hi]
    extern __shared__ int sh[];
    int* key = sh;
    int* snode = sh + P_hi;
    int* pos = snode + P_hi;
    int* runid = pos + P_hi;
    const int row = blockIdx.x;
    const int slot = row >> 3, o = row & 7;
    const int el = slot_el[slot];
    const double zero[3] = {0.0, 0.0, 0.0};
    for (int n = threadIdx.x; n < P_hi; n += blockDim.x)
    {
        double y[3], s[3];
        node_position(PG, el, n, hi_nodes, zero, pH, y);
        const double p0 = y[0] - off[3 * o], p1 = y[1] - off[3 * o + 1], p2 = y[2] - off[3 * o + 2];
        cart_to_interp(p0, p1, p2, cH, s);
        const int fe = element_for_point(s, CG.dmin, CG.dmax, CG.hfi, CG.nf);
        key[n] = fe < 0 ? 0x7fffffff : fe;
    }
    __syncthreads();
    for (int n = threadIdx.x; n < P_hi; n += blockDim.x)
    {
        const int kn = key[n];
        int rank = 0;
        for (int m = 0; m < P_hi; m++)
        {
            const int km = key[m];
            rank += (km < kn) || (km == kn && m < n);
        }
        snode[rank] = n;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int off_run = 0, start = 0, nrun = 0;
        for (int i = 0; i <= P_hi; i++)
        {
            const bool end = i == P_hi || key[snode[i]] != key[snode[start]];
            if (end)
            {
                if (key[snode[start]] == 0x7fffffff)
                    break; // the nodes outside the domain sort last and are dropped
                const int len = i - start;
                for (int j = 0; j < len; j++)
                {
                    pos[start + j] = off_run + j;
                    runid[start + j] = nrun;
                }
                if (fill && nrun < fe_pad)
                    fe_list[(size_t)row * (fe_pad + 1) + nrun] =
                        make_int2(key[snode[start]], off_run / UPGEO_RUN);
                nrun++;
                off_run += (len + UPGEO_RUN - 1) / UPGEO_RUN * UPGEO_RUN;
                start = i;
            }
            if (i < P_hi && key[snode[i]] == 0x7fffffff)
            {
                for (int j = i; j < P_hi; j++)
                    pos[j] = -1;
                break;
            }
        }
        if (!fill)
        {
            row_len[2 * row] = off_run;
            row_len[2 * row + 1] = nrun;
        }
        else if (nrun <= fe_pad)
            // sentinel after the last run: (-1, groups of the row)
            fe_list[(size_t)row * (fe_pad + 1) + nrun] = make_int2(-1, off_run / UPGEO_RUN);
    }
    __syncthreads();
    if (!fill)
        return;
    // entry (group g, member r) lives at r * (P_pad / UPGEO_RUN) + g, so the
    // threads of a warp (consecutive groups) read consecutive entries
    const size_t base = (size_t)row * P_pad;
    const int ngroups = P_pad / UPGEO_RUN;
    for (int i = threadIdx.x; i < P_hi; i += blockDim.x)
    {
        if (pos[i] < 0)
            continue;
        const size_t at = base + (size_t)(pos[i] % UPGEO_RUN) * ngroups + pos[i] / UPGEO_RUN;
        const int n = snode[i];
        double y[3], s[3];
        node_position(PG, el, n, hi_nodes, zero, pH, y);
        const double dp2 = y[0] * y[0] + y[1] * y[1] + y[2] * y[2];
        const double p0 = y[0] - off[3 * o], p1 = y[1] - off[3 * o + 1], p2 = y[2] - off[3 * o + 2];
        cart_to_interp(p0, p1, p2, cH, s);
        UpGeo64 g;
        g.fe = key[n];
        g.node = n;
        to_local(g.fe, s, CG.dmin, CG.hf, CG.hfi, CG.nf, g.loc);
        if (fill == 2)
        {
            // distance table: d - d_parent and d_parent / d for every wavenumber
            const double d = sqrt(p0 * p0 + p1 * p1 + p2 * p2), dp = sqrt(dp2);
            g.tr = d - dp;
            g.ti = dp / d;
        }
        else
        {
            const cplx<double> tf = P::transfer(p0 * p0 + p1 * p1 + p2 * p2, dp2, kp);
            g.tr = tf.re;
            g.ti = tf.im;
            g64[at] = g;
        }
        UpGeo32 h;
        h.fe = g.fe;
        h.node = n;
        h.pad = runid[i];
        h.loc[0] = (float)g.loc[0];
        h.loc[1] = (float)g.loc[1];
        h.loc[2] = (float)g.loc[2];
        h.tr = (float)g.tr;
        h.ti = (float)g.ti;
        g32[at] = h;
    }
}

template <int KIND>
int upgeo_row_max(const LevelGeom& PG, const LevelGeom& CG, double pH, double cH,
                  const double* off_dev, const int* slot_el, int n_slots, const double* hi_nodes,
                  int P_hi, KParams kp, int* row_len_dev, int* row_len_host, int* runs_max)
{
    *runs_max = 0;
    if (n_slots <= 0)
        return 0;
    build_upgeo_kernel<KIND><<<n_slots * 8, 256, 4 * P_hi * sizeof(int)>>>(
        PG, CG, pH, cH, off_dev, slot_el, hi_nodes, P_hi, kp, 0, 0, row_len_dev, nullptr, nullptr,
        0, nullptr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpy(row_len_host, row_len_dev, (size_t)n_slots * 16 * sizeof(int),
                       cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        throw Error(2, std::string("build_upgeo_kernel: ") + cudaGetErrorString(e));
    int mx = 0, rx = 0;
    for (int i = 0; i < n_slots * 8; i++)
    {
        mx = row_len_host[2 * i] > mx ? row_len_host[2 * i] : mx;
        rx = row_len_host[2 * i + 1] > rx ? row_len_host[2 * i + 1] : rx;
    }
    *runs_max = rx;
    return mx;
}

template <int KIND>
void launch_build_upgeo(const LevelGeom& PG, const LevelGeom& CG, double pH, double cH,
                        const double* off_dev, const int* slot_el, int n_slots,
                        const double* hi_nodes, int P_hi, KParams kp, int P_pad, UpGeo64* g64,
                        UpGeo32* g32, int fe_pad, int2* fe_list)
{
    if (n_slots <= 0 || P_pad <= 0)
        return;
    // without an FP64 table (g64 null): the distance table
    build_upgeo_kernel<KIND><<<n_slots * 8, 256, 4 * P_hi * sizeof(int)>>>(
        PG, CG, pH, cH, off_dev, slot_el, hi_nodes, P_hi, kp, g64 ? 1 : 2, P_pad, nullptr, g64,
        g32, fe_pad, fe_list);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        throw Error(2, std::string("build_upgeo_kernel: ") + cudaGetErrorString(e));
}


struct C2FArgs
{
    LevelGeom G;
    const int* __restrict__ idx; // coarse cones to refine (null: all of the level)
    // batched right-hand sides (fixed-order kernel): blockIdx.y selects the plane
    long long cv_plane, fc_plane;
    const int* __restrict__ cc_box;
    const int* __restrict__ cc_el;
    const double2* __restrict__ cvals;
    const double* __restrict__ A; // A0 | A1 | A2, row-major (f_d lo_d) x ho_d
    const int* __restrict__ fmap;
    double2* fcoef;
    int hi[3], lo[3], f[3];
    int P_hi, P_lo;
};

// Coarse nodal values -> fine Chebyshev coefficients of the active sub-cones.
static __global__ void __launch_bounds__(256) coarse_to_fine_kernel(C2FArgs a)
{
    extern __shared__ double2 s2[];
    const int c = a.idx ? a.idx[blockIdx.x] : (int)blockIdx.x;
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
    for (int o = threadIdx.x; o < F0 * h1 * h2; o += blockDim.x)
    {
        const int i0 = o % F0, r = o / F0;
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
            a.fcoef[(size_t)gf * a.P_lo + q] = B2[(j0 * lo0 + i0) + F0 * ((j1 * lo1 + i1) + F1 * i2)];
        }
    }
}

struct EvalArgs
{
    const LevelGeom* __restrict__ lv;
    int L; // levels
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
    double* out;     // complex (interleaved) or real for Laplace
    double2* unear;  // near-field sums per sorted target (written by the near pass)
    int real_out;
    unsigned long long* err;
    int P_lo;
    int lo[3];
    KParams kp;
};

constexpr int EVAL_THREADS = 128;
// Threads of the far-field evaluation: 256 leave fewer lanes idle than 128 on
// target leaves whose size does not divide the block (leaves of 17-69
// targets at N = 1e6: 89 % of lanes busy against 77 %).
constexpr int FAR_THREADS = 256;
constexpr int EVAL_NEAR = 0, EVAL_FAR = 1; // the two passes of target evaluation

// One CTA per target leaf.  A leaf holds fewer targets than threads, so
// thread (ti, si) takes target ti and every S-th near source / far box
// (S = threads / targets); the S partial sums are added in a fixed order.
template <int KIND, int N0, int N1, int N2, int PART>
__global__ void __launch_bounds__(EVAL_THREADS) target_eval_kernel(EvalArgs a)
{
    using P = Plugin<KIND>;
    __shared__ double xs[EVAL_THREADS], ys[EVAL_THREADS], zs[EVAL_THREADS];
    __shared__ double wr[EVAL_THREADS], wi[EVAL_THREADS];
    __shared__ double n0[P::needs_normals ? EVAL_THREADS : 1], n1[P::needs_normals ? EVAL_THREADS : 1],
        n2[P::needs_normals ? EVAL_THREADS : 1];
    __shared__ double rr[EVAL_THREADS], ri[EVAL_THREADS];
    const int tl = blockIdx.x;
    const int tf = a.tl_first[tl], tlast = a.tl_last[tl];
    const long long nb0 = a.near_off[tl], nb1 = PART == EVAL_NEAR ? a.near_off[tl + 1] : nb0;
    const long long fb0 = a.far_off[tl], fb1 = PART == EVAL_FAR ? a.far_off[tl + 1] : fb0;
    for (int base = tf; base < tlast; base += EVAL_THREADS)
    {
        const int cnt = min(EVAL_THREADS, tlast - base);
        const int S = EVAL_THREADS / cnt;
        const int ti = threadIdx.x % cnt, si = threadIdx.x / cnt;
        const bool active = si < S;
        const int t = base + ti;
        const double y0 = a.tx[t], y1 = a.ty[t], y2 = a.tz[t];
        cplx<double> acc = {0.0, 0.0};
        for (long long e = nb0; e < nb1; e++)
        {
            const int sb = a.near_src[e];
            const int sf = a.T.box_first[sb], sl = a.T.box_last[sb];
            for (int cs = sf; cs < sl; cs += EVAL_THREADS)
            {
                const int ccnt = min(EVAL_THREADS, sl - cs);
                __syncthreads();
                if (threadIdx.x < ccnt)
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
                if (active)
                    for (int i = si; i < ccnt; i += S)
                    {
                        const double x[3] = {xs[i] - y0, ys[i] - y1, zs[i] - y2};
                        const double nv[3] = {P::needs_normals ? n0[i] : 0.0,
                                              P::needs_normals ? n1[i] : 0.0,
                                              P::needs_normals ? n2[i] : 0.0};
                        cfma(acc, cplx<double>{wr[i], wi[i]}, P::kernel(x, nv, a.kp));
                    }
            }
        }
        if (active)
            for (long long e = fb0 + si; e < fb1; e += S)
            {
                const int sb = a.far_src[e];
                const LevelGeom& G = a.lv[a.T.box_level[sb]];
                const double p[3] = {y0 - a.T.box_c[3 * sb], y1 - a.T.box_c[3 * sb + 1],
                                     y2 - a.T.box_c[3 * sb + 2]};
                double s[3], loc[3];
                cart_to_interp(p[0], p[1], p[2], a.T.box_H[sb], s);
                const int fe = element_for_point(s, G.dmin, G.dmax, G.hfi, G.nf);
                if (fe < 0)
                    continue;
                const long long nft = (long long)G.nf[0] * G.nf[1] * G.nf[2];
                const int gf = a.fmap[G.fmap_off + (long long)(sb - G.box_off) * nft + fe];
                if (gf < 0)
                {
                    atomicAdd(a.err, 1ull);
                    continue;
                }
                to_local(fe, s, G.dmin, G.hf, G.hfi, G.nf, loc);
                const cplx<double> v = Cheb<N0, N1, N2>::eval(a.fcoef + (size_t)gf * a.P_lo, loc, a.lo);
                cfma(acc, v, P::cf(p, a.kp));
            }
        __syncthreads();
        rr[threadIdx.x] = acc.re;
        ri[threadIdx.x] = acc.im;
        __syncthreads();
        if (active && si == 0)
        {
            double sr = 0, sim = 0;
            for (int s = 0; s < S; s++)
            {
                sr += rr[ti + s * cnt];
                sim += ri[ti + s * cnt];
            }
            if (PART == EVAL_NEAR)
                a.unear[t] = make_double2(sr, sim);
            else
            {
                const double2 nr = a.unear[t];
                sr += nr.x;
                sim += nr.y;
                const long long o = a.tgt_perm[t];
                if (a.real_out)
                    a.out[o] = sr;
                else
                {
                    a.out[2 * o] = sr;
                    a.out[2 * o + 1] = sim;
                }
            }
        }
    }
}

// FP64 direct sum at selected targets: one CTA per target, Kahan-compensated
// per-thread partial sums, then a pairwise block reduction.
template <int KIND>
__global__ void __launch_bounds__(256) direct_eval_kernel(SrcArgs S, const double2* __restrict__ w,
                                                          long long ns, const double* __restrict__ tx,
                                                          const double* __restrict__ ty,
                                                          const double* __restrict__ tz,
                                                          const int* __restrict__ tpos, KParams kp,
                                                          double2* out)
{
    using P = Plugin<KIND>;
    __shared__ double sr[256], si[256];
    const int j = tpos[blockIdx.x];
    const double y0 = tx[j], y1 = ty[j], y2 = tz[j];
    double ar = 0, ai = 0, cr = 0, ci = 0;
    for (long long s = threadIdx.x; s < ns; s += blockDim.x)
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

// ===========================================================================
// Mixed-precision variants.  Buffers are reused as float2: permuted
// densities, coarse nodal values and fine coefficients in FP32.
// ===========================================================================
// Loads of FP32 coefficient rows (N0 consecutive float2) as 16-byte vectors:
// one row when N0 is even, two rows when N0 is odd and N1 even (the pair
// then starts on a 16-byte boundary), else one float2 at a time.  Blocks
// start on 16-byte boundaries whenever N0 N1 N2 is even.  SHARED selects
// plain loads (shared memory) instead of read-only global loads.
template <int N0, int N1, bool SHARED = false> struct CoefRows
{
    static constexpr bool VEC = (N0 % 2 == 0) || (N1 % 2 == 0);
    static constexpr int ROWS = (N0 % 2 == 0) ? 1 : (N1 % 2 == 0 ? 2 : 1);
    __device__ static __forceinline__ void load(const float2* __restrict__ p, float2* v)
    {
        if constexpr (VEC)
        {
            const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
            for (int h = 0; h < ROWS * N0 / 2; h++)
            {
                const float4 u = SHARED ? q[h] : __ldg(q + h);
                v[2 * h] = make_float2(u.x, u.y);
                v[2 * h + 1] = make_float2(u.z, u.w);
            }
        }
        else
        {
#pragma unroll
            for (int h = 0; h < ROWS * N0; h++)
                v[h] = SHARED ? p[h] : __ldg(p + h);
        }
    }
};

// SHARED: c points into shared memory (plain loads); else read-only global.
template <int N0, int N1, int N2, bool SHARED = false> struct ChebF
{
    __device__ static __forceinline__ cplx<float> eval(const float2* __restrict__ c, const float* x,
                                                       const int*)
    {
        float t0[N0], t1[N1], t2[N2];
        t0[0] = t1[0] = t2[0] = 1.f;
        if (N0 > 1)
            t0[1] = x[0];
        if (N1 > 1)
            t1[1] = x[1];
        if (N2 > 1)
            t2[1] = x[2];
#pragma unroll
        for (int i = 2; i < N0; i++)
            t0[i] = fmaf(2.f * x[0], t0[i - 1], -t0[i - 2]);
#pragma unroll
        for (int i = 2; i < N1; i++)
            t1[i] = fmaf(2.f * x[1], t1[i - 1], -t1[i - 2]);
#pragma unroll
        for (int i = 2; i < N2; i++)
            t2[i] = fmaf(2.f * x[2], t2[i - 1], -t2[i - 2]);
        // T_0 = 1: every sum starts from its first term
        float ar, ai;
#pragma unroll
        for (int k = 0; k < N2; k++)
        {
            float br, bi;
#pragma unroll
            for (int j = 0; j < N1; j += CoefRows<N0, N1>::ROWS)
            {
                float2 v[CoefRows<N0, N1>::ROWS * N0];
                CoefRows<N0, N1, SHARED>::load(c + N0 * (j + N1 * k), v);
#pragma unroll
                for (int jj = 0; jj < CoefRows<N0, N1>::ROWS; jj++)
                {
                    float cr = v[jj * N0].x, ci = v[jj * N0].y;
#pragma unroll
                    for (int i = 1; i < N0; i++)
                    {
                        cr = fmaf(v[jj * N0 + i].x, t0[i], cr);
                        ci = fmaf(v[jj * N0 + i].y, t0[i], ci);
                    }
                    if (j + jj == 0)
                        br = cr, bi = ci;
                    else
                    {
                        br = fmaf(cr, t1[j + jj], br);
                        bi = fmaf(ci, t1[j + jj], bi);
                    }
                }
            }
            if (k == 0)
                ar = br, ai = bi;
            else
            {
                ar = fmaf(br, t2[k], ar);
                ai = fmaf(bi, t2[k], ai);
            }
        }
        return {ar, ai};
    }
};

template <> struct ChebF<0, 0, 0, false>
{
    __device__ static __forceinline__ cplx<float> eval(const float2* __restrict__ c, const float* x,
                                                       const int* n)
    {
        float t0[16], t1[16], t2[16];
        float* ts[3] = {t0, t1, t2};
        for (int d = 0; d < 3; d++)
        {
            ts[d][0] = 1.f;
            if (n[d] > 1)
                ts[d][1] = x[d];
            for (int i = 2; i < n[d]; i++)
                ts[d][i] = fmaf(2.f * x[d], ts[d][i - 1], -ts[d][i - 2]);
        }
        float ar = 0, ai = 0;
        int q = 0;
        for (int k = 0; k < n[2]; k++)
        {
            float br = 0, bi = 0;
            for (int j = 0; j < n[1]; j++)
            {
                float cr = 0, ci = 0;
                for (int i = 0; i < n[0]; i++, q++)
                {
                    const float2 v = __ldg(c + q);
                    cr = fmaf(v.x, t0[i], cr);
                    ci = fmaf(v.y, t0[i], ci);
                }
                br = fmaf(cr, t1[j], br);
                bi = fmaf(ci, t1[j], bi);
            }
            ar = fmaf(br, t2[k], ar);
            ai = fmaf(bi, t2[k], ai);
        }
        return {ar, ai};
    }
};

// Fine cone of the point p (difference to the box centre, FP64) in a box of
// side H: FP32 angles first; when they land outside the domain or in an
// inactive cone, the lookup is redone in FP64, the arithmetic the active-cone
// tables were built with.  Returns the global fine cone (or -1 when the point
// is outside the domain) and the local coordinates.
__device__ __forceinline__ int fine_lookup_mixed(const LevelGeom& G, const int* __restrict__ fm,
                                                 const double* p, double H, float* loc,
                                                 unsigned long long* err)
{
    float sf[3];
    cart_to_interp_f((float)p[0], (float)p[1], (float)p[2], (float)H, sf);
    int fe = -1;
    {
        bool inside = true;
        int id = 0, stride = 1;
#pragma unroll
        for (int j = 0; j < 3; j++)
        {
            const float lo = (float)G.dmin[j], hi = (float)G.dmax[j];
            inside = inside && sf[j] >= lo && sf[j] <= hi;
            int q = (int)floorf((sf[j] - lo) * (float)G.hfi[j]);
            q = min(max(q, 0), G.nf[j] - 1);
            id += q * stride;
            stride *= G.nf[j];
        }
        if (inside)
            fe = id;
    }
    int gf = fe >= 0 ? fm[fe] : -1;
    if (gf >= 0)
    {
        int r = fe;
        const int i0 = r % G.nf[0];
        r /= G.nf[0];
        const int i1 = r % G.nf[1], i2 = r / G.nf[1];
        const int idx[3] = {i0, i1, i2};
#pragma unroll
        for (int d = 0; d < 3; d++)
        {
            const float a2 = 2.f * (float)G.hfi[d];
            const float b = (float)(G.dmin[d] + ((double)idx[d] + 0.5) * G.hf[d]);
            loc[d] = (sf[d] - b) * a2;
        }
        return gf;
    }
    double s[3], ld[3];
    cart_to_interp(p[0], p[1], p[2], H, s);
    fe = element_for_point(s, G.dmin, G.dmax, G.hfi, G.nf);
    if (fe < 0)
        return -1;
    gf = fm[fe];
    if (gf < 0)
    {
        atomicAdd(err, 1ull);
        return -1;
    }
    to_local(fe, s, G.dmin, G.hf, G.hfi, G.nf, ld);
    loc[0] = (float)ld[0];
    loc[1] = (float)ld[1];
    loc[2] = (float)ld[2];
    return gf;
}


static __global__ void permute_weights_mixed_kernel(const double* __restrict__ in, int real_in,
                                                    const long long* __restrict__ perm, float2* w,
                                                    long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
    {
        const long long j = perm[i];
        if (real_in)
            w[i] = make_float2((float)in[j], 0.f);
        else
        {
            const double2 v = reinterpret_cast<const double2*>(in)[j];
            w[i] = make_float2((float)v.x, (float)v.y);
        }
    }
}

template <int KIND>
__global__ void __launch_bounds__(NODE_THREADS) leaf_sample_mixed_kernel(LeafArgs a)
{
    using P = PluginF<KIND>;
    extern __shared__ float smf[];
    const int c = a.idx[blockIdx.x];
    const int node0 = blockIdx.y * NPT * blockDim.x;
    const int box = a.cc_box[c], el = a.cc_el[c];
    const double xc[3] = {a.T.box_c[3 * box], a.T.box_c[3 * box + 1], a.T.box_c[3 * box + 2]};
    const double H = a.T.box_H[box];
    const float2* wf = reinterpret_cast<const float2*>(a.w);
    float b[NPT][3], dc[NPT];
    cplx<float> acc[NPT];
#pragma unroll
    for (int q = 0; q < NPT; q++)
    {
        const int n = node0 + threadIdx.x + q * blockDim.x;
        acc[q] = {0.f, 0.f};
        b[q][0] = b[q][1] = b[q][2] = 0.f;
        dc[q] = 1.f;
        if (n < a.P_hi)
        {
            double y[3];
            node_position(a.G, el, n, a.hi_nodes, xc, H, y);
            const double e0 = y[0] - xc[0], e1 = y[1] - xc[1], e2 = y[2] - xc[2];
            b[q][0] = (float)e0;
            b[q][1] = (float)e1;
            b[q][2] = (float)e2;
            dc[q] = (float)sqrt(e0 * e0 + e1 * e1 + e2 * e2);
        }
    }
    const int nt = blockDim.x;
    float* ax = smf;
    float* ay = ax + nt;
    float* az = ay + nt;
    float* wr = az + nt;
    float* wi = wr + nt;
    float* n0 = wi + nt;
    float* n1 = n0 + nt;
    float* n2 = n1 + nt;
    float* aa = n2 + nt;
    const int f = a.T.box_first[box], l = a.T.box_last[box];
    for (int cs = f; cs < l; cs += nt)
    {
        const int cnt = min(nt, l - cs);
        __syncthreads();
        if (threadIdx.x < cnt)
        {
            const int i = cs + threadIdx.x;
            const double a0 = a.S.sx[i] - xc[0], a1 = a.S.sy[i] - xc[1], a2 = a.S.sz[i] - xc[2];
            ax[threadIdx.x] = (float)a0;
            ay[threadIdx.x] = (float)a1;
            az[threadIdx.x] = (float)a2;
            aa[threadIdx.x] = (float)(a0 * a0 + a1 * a1 + a2 * a2);
            const float2 wv = wf[i];
            wr[threadIdx.x] = wv.x;
            wi[threadIdx.x] = wv.y;
            if (P::needs_normals)
            {
                n0[threadIdx.x] = (float)a.S.nx[i];
                n1[threadIdx.x] = (float)a.S.ny[i];
                n2[threadIdx.x] = (float)a.S.nz[i];
            }
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < NPT; q++)
        {
            if (node0 + threadIdx.x + q * blockDim.x >= a.P_hi)
                continue;
            for (int i = 0; i < cnt; i++)
            {
                const float av[3] = {ax[i], ay[i], az[i]};
                const float nv[3] = {P::needs_normals ? n0[i] : 0.f, P::needs_normals ? n1[i] : 0.f,
                                     P::needs_normals ? n2[i] : 0.f};
                const cplx<float> v = P::factored(av, aa[i], b[q], nv, {wr[i], wi[i]}, dc[q], a.kp);
                acc[q].re += v.re;
                acc[q].im += v.im;
            }
        }
    }
    float2* cv = reinterpret_cast<float2*>(a.cvals);
#pragma unroll
    for (int q = 0; q < NPT; q++)
    {
        const int n = node0 + threadIdx.x + q * blockDim.x;
        if (n < a.P_hi)
            cv[(size_t)c * a.P_hi + n] = make_float2(acc[q].re, acc[q].im);
    }
}

// Chebyshev sums of R points sharing one coefficient block: every coefficient
// is loaded once and used R times.  N0 = 0 selects the runtime-order path.
template <typename T> struct VecOf;
template <> struct VecOf<double>
{
    using type = double2;
};
template <> struct VecOf<float>
{
    using type = float2;
};

template <typename T, int N> __device__ __forceinline__ void cheb_basis(T x, T* t)
{
    t[0] = T(1);
    if (N > 1)
        t[1] = x;
#pragma unroll
    for (int i = 2; i < N; i++)
        t[i] = fma(T(2) * x, t[i - 1], -t[i - 2]);
}

template <typename T, int N0, int N1, int N2, int R, bool SHARED = false> struct ChebMulti
{
    using V = typename VecOf<T>::type;
    // SHARED: c points into shared memory (plain loads); else read-only
    // global.  FP32 rows are read as 16-byte vectors (CoefRows).
    static constexpr int ROWS = std::is_same<T, float>::value ? CoefRows<N0, N1>::ROWS : 1;
    __device__ static __forceinline__ void load_rows(const V* __restrict__ c, V* v)
    {
        if constexpr (std::is_same<T, float>::value)
            CoefRows<N0, N1, SHARED>::load(c, v);
        else
        {
#pragma unroll
            for (int i = 0; i < N0; i++)
                v[i] = SHARED ? c[i] : __ldg(c + i);
        }
    }
    __device__ static __forceinline__ void eval(const V* __restrict__ c, const T (&x)[R][3],
                                                const int*, T (&ore)[R], T (&oim)[R])
    {
        T t0[R][N0], t1[R][N1], t2[R][N2];
#pragma unroll
        for (int r = 0; r < R; r++)
        {
            cheb_basis<T, N0>(x[r][0], t0[r]);
            cheb_basis<T, N1>(x[r][1], t1[r]);
            cheb_basis<T, N2>(x[r][2], t2[r]);
        }
        // T_0 = 1: every sum starts from its first term instead of adding
        // it to zero (the same values; one instruction less per sum)
#pragma unroll
        for (int k = 0; k < N2; k++)
        {
            T br[R], bi[R];
#pragma unroll
            for (int j = 0; j < N1; j += ROWS)
            {
                V v[ROWS * N0];
                load_rows(c + N0 * (j + N1 * k), v);
#pragma unroll
                for (int jj = 0; jj < ROWS; jj++)
                {
                    T cr[R], ci[R];
#pragma unroll
                    for (int r = 0; r < R; r++)
                    {
                        cr[r] = v[jj * N0].x;
                        ci[r] = v[jj * N0].y;
                    }
#pragma unroll
                    for (int i = 1; i < N0; i++)
                    {
#pragma unroll
                        for (int r = 0; r < R; r++)
                        {
                            cr[r] = fma(v[jj * N0 + i].x, t0[r][i], cr[r]);
                            ci[r] = fma(v[jj * N0 + i].y, t0[r][i], ci[r]);
                        }
                    }
#pragma unroll
                    for (int r = 0; r < R; r++)
                    {
                        if (j + jj == 0)
                            br[r] = cr[r], bi[r] = ci[r];
                        else
                        {
                            br[r] = fma(cr[r], t1[r][j + jj], br[r]);
                            bi[r] = fma(ci[r], t1[r][j + jj], bi[r]);
                        }
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < R; r++)
            {
                if (k == 0)
                    ore[r] = br[r], oim[r] = bi[r];
                else
                {
                    ore[r] = fma(br[r], t2[r][k], ore[r]);
                    oim[r] = fma(bi[r], t2[r][k], oim[r]);
                }
            }
        }
    }
};

template <int R> struct ChebMulti<double, 0, 0, 0, R, false>
{
    __device__ static __forceinline__ void eval(const double2* __restrict__ c,
                                                const double (&x)[R][3], const int* n,
                                                double (&ore)[R], double (&oim)[R])
    {
        for (int r = 0; r < R; r++)
        {
            const cplx<double> v = cheb_eval3<16>(c, x[r], n);
            ore[r] = v.re;
            oim[r] = v.im;
        }
    }
};

template <int R> struct ChebMulti<float, 0, 0, 0, R, false>
{
    __device__ static __forceinline__ void eval(const float2* __restrict__ c,
                                                const float (&x)[R][3], const int* n,
                                                float (&ore)[R], float (&oim)[R])
    {
        for (int r = 0; r < R; r++)
        {
            const cplx<float> v = ChebF<0, 0, 0>::eval(c, x[r], n);
            ore[r] = v.re;
            oim[r] = v.im;
        }
    }
};

constexpr int UP_THREADS = 128;
constexpr size_t UP_STAGED_SMEM_MAX = 96 * 1024;

// One CTA per coarse cone of a box with children (CTAs ordered by cone
// element, so consecutive CTAs share their geometry-table rows in L2).  For
// every child, the cone's nodes inside the child's domain come from the
// level's geometry table in groups of R sharing one child cone: one
// coefficient gather serves R nodes.  Each node is updated once per child,
// so the per-node sums in shared memory need no atomics.
template <int KIND, int N0, int N1, int N2>
__global__ void __launch_bounds__(UP_THREADS) upward_kernel(UpArgs a)
{
    constexpr int R = 2;
    extern __shared__ double2 acc64[];
    const int c = a.idx[blockIdx.x];
    const int slot = a.slot[blockIdx.x];
    const int box = a.cc_box[c], el = a.cc_el[c];
    for (int n = threadIdx.x; n < a.P_hi; n += blockDim.x)
        acc64[n] = make_double2(0.0, 0.0);
    const LevelGeom& C = a.GC;
    const long long nf = (long long)C.nf[0] * C.nf[1] * C.nf[2];
    for (int o = 0; o < 8; o++)
    {
        const int cb = a.T.box_child[8 * box + o];
        if (cb < 0)
            continue;
        __syncthreads();
        const int* fm = a.fmap + C.fmap_off + (long long)(cb - C.box_off) * nf;
        const UpGeo64* row = a.geo64 + ((size_t)slot * 8 + o) * a.P_pad;
        const int ngroups = a.P_pad / UPGEO_RUN;
        // a table group holds UPGEO_RUN entries; FP64 evaluates it as pairs
        for (int gh = threadIdx.x; gh < ngroups * (UPGEO_RUN / R); gh += blockDim.x)
        {
            const int g = gh % ngroups, h = gh / ngroups;
            UpGeo64 e[R];
#pragma unroll
            for (int r = 0; r < R; r++)
                e[r] = row[(size_t)(h * R + r) * ngroups + g];
            if (e[0].fe < 0)
                continue;
            const int gf = fm[e[0].fe];
            if (gf < 0)
            {
#pragma unroll
                for (int r = 0; r < R; r++)
                {
                    cplx<double> v;
                    if (e[r].node >= 0 &&
                        upward_fallback64<KIND, N0, N1, N2>(a, box, el, e[r].node, cb, fm, v))
                    {
                        acc64[e[r].node].x += v.re;
                        acc64[e[r].node].y += v.im;
                    }
                }
                continue;
            }
            double x[R][3], vr[R], vi[R];
#pragma unroll
            for (int r = 0; r < R; r++)
                for (int d = 0; d < 3; d++)
                    x[r][d] = e[r].loc[d];
            ChebMulti<double, N0, N1, N2, R>::eval(a.fcoef + (size_t)gf * a.P_lo, x, a.lo, vr, vi);
#pragma unroll
            for (int r = 0; r < R; r++)
                if (e[r].node >= 0)
                {
                    const double2 s = acc64[e[r].node];
                    acc64[e[r].node] = make_double2(s.x + (vr[r] * e[r].tr - vi[r] * e[r].ti),
                                                    s.y + (vr[r] * e[r].ti + vi[r] * e[r].tr));
                }
        }
    }
    __syncthreads();
    for (int n = threadIdx.x; n < a.P_hi; n += blockDim.x)
        a.cvals[(size_t)c * a.P_hi + n] = acc64[n];
}

// Stride (in float2) of a staged coefficient block: at least P_lo, a
// multiple of 2 (16-byte rows for cp.async) and 2 mod 4, so that the blocks
// of eight consecutive runs start in eight different bank pairs.
__host__ __device__ constexpr int up_block_stride(int p_lo)
{
    return p_lo + ((2 - p_lo % 4) + 4) % 4;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Shared memory of the staged upward kernel staging rch runs at a time:
// the parent's accumulators, rch coefficient blocks, and per child the fine
// cone and first group of each of its fe_pad + 1 run-list entries plus the
// row's run and group counts.
template <int N0, int N1, int N2>
size_t upward_staged_smem(int P_hi, int rch, int fe_pad)
{
    constexpr int P_LO = N0 * N1 * N2;
    return ((size_t)((P_hi + 1) & ~1) + (size_t)rch * up_block_stride(P_LO)) * sizeof(float2) +
           ((size_t)16 * (fe_pad + 1) + 16) * sizeof(int);
}

// Runs staged at a time: all of a row's runs when they fit in about 16 KB
// (rows average a handful of runs; the longest ones take several chunks).
template <int N0, int N1, int N2>
int upward_staged_rch(int fe_pad)
{
    constexpr int per = up_block_stride(N0 * N1 * N2) * (int)sizeof(float2);
    const int fit = 16 * 1024 / per;
    return fe_pad < fit ? fe_pad : (fit > 0 ? fit : 1);
}

// Threads of the staged upward kernel: an average geometry row has a few
// dozen groups, so small CTAs keep most threads busy.
constexpr int UPS_THREADS = 64;

// Mixed-precision upward transfer with the coefficient blocks in shared
// memory.  Per child, every run of the (slot, octant) geometry row needs one
// child fine cone; its block (P_lo coefficients) is copied once into shared
// memory with cp.async (one warp per block), rch runs at a time, after which
// the Chebyshev sums of those runs' groups read only shared memory.  The
// fine cones of all eight children's runs are looked up together when the
// block starts (one pass of independent loads), so a chunk's copies start
// without a chain of dependent global loads.
// Compile-time orders only (P_lo even, so that a block is a whole number of
// 16-byte chunks).
// MK: every plane (blockIdx.y) has its own wavenumber; the centre-shift
// factor is formed from the distance table per plane.
// At least 8 CTAs per SM (128 registers; measured at N = 1e6, p = 9: levels
// 2 and 3 of the batched matvec 0.79 + 3.45 ms with 8 or 7, 0.86 + 3.71 with
// 10 (96 registers, more spills), 0.85 + 3.66 with 6, 0.93 + 4.09 with 12).
template <int KIND, int N0, int N1, int N2, bool MK = false>
__global__ void __launch_bounds__(UPS_THREADS, 8) upward_staged_kernel(UpArgs a)
{
    constexpr int R = UPGEO_RUN;
    constexpr int P_LO = N0 * N1 * N2;
    constexpr int BS = up_block_stride(P_LO);
    constexpr int CH = P_LO * (int)sizeof(float2) / 16; // 16-byte chunks per block
    static_assert(P_LO % 2 == 0, "staged blocks need an even number of coefficients");
    extern __shared__ __align__(16) float2 up_sh[];
    float2* acc = up_sh;
    float2* blk = up_sh + ((a.P_hi + 1) & ~1);
    const int FL = a.fe_pad + 1;
    int* run_gf = reinterpret_cast<int*>(blk + (size_t)a.rch * BS); // [8][FL] child fine cone
    int* run_g = run_gf + 8 * FL;                                   // [8][FL] first group
    int* row_n = run_g + 8 * FL; // [8] runs of the row, [8] groups of the row
    const int c = a.idx[blockIdx.x];
    const int slot = a.slot[blockIdx.x];
    const int box = a.cc_box[c], el = a.cc_el[c];
    const float2* fcf = reinterpret_cast<const float2*>(a.fcoef) + blockIdx.y * a.fc_plane;
    const int warp = threadIdx.x >> 5;
    const int ngroups = a.P_pad / R;
    for (int n = threadIdx.x; n < a.P_hi; n += blockDim.x)
        acc[n] = make_float2(0.f, 0.f);
    if (threadIdx.x < 8)
    {
        row_n[threadIdx.x] = a.fe_pad;
        row_n[8 + threadIdx.x] = ngroups;
    }
    __syncthreads();
    const LevelGeom& C = a.GC;
    const long long nf = (long long)C.nf[0] * C.nf[1] * C.nf[2];
    for (int i = threadIdx.x; i < 8 * FL; i += blockDim.x)
    {
        const int o = i / FL, r = i - o * FL;
        const int cb = a.T.box_child[8 * box + o];
        const int2 f = a.fe_list[((size_t)slot * 8 + o) * FL + r];
        run_gf[i] = cb >= 0 && f.x >= 0 ? a.fmap[C.fmap_off + (long long)(cb - C.box_off) * nf + f.x]
                                        : -1;
        run_g[i] = f.y;
        if (f.x < 0 && f.y >= 0)
        {
            // the sentinel after the row's last run: (-1, groups of the row)
            row_n[o] = r;
            row_n[8 + o] = f.y;
        }
    }
    __syncthreads();
    for (int o = 0; o < 8; o++)
    {
        const int cb = a.T.box_child[8 * box + o];
        if (cb < 0)
            continue;
        const int* fm = a.fmap + C.fmap_off + (long long)(cb - C.box_off) * nf;
        const int* rgf = run_gf + o * FL;
        const UpGeo32* row = a.geo32 + ((size_t)slot * 8 + o) * a.P_pad;
        const int nrun = row_n[o];
        for (int r0 = 0; r0 < nrun; r0 += a.rch)
        {
            const int r1 = min(r0 + a.rch, nrun);
            // the next run's first group, or the row's end
            const int g_end = r1 < nrun ? run_g[o * FL + r1] : row_n[8 + o];
            __syncthreads(); // the previous runs' blocks are no longer read
            for (int r = r0 + warp; r < r1; r += UPS_THREADS / 32)
            {
                const int gf = rgf[r];
                if (gf < 0)
                    continue;
                const float2* src = fcf + (size_t)gf * P_LO;
                float2* dst = blk + (size_t)(r - r0) * BS;
                for (int ch = threadIdx.x & 31; ch < CH; ch += 32)
                    cp_async16(dst + 2 * ch, src + 2 * ch);
            }
            // the first group's table entries load while the blocks arrive
            const int g0 = run_g[o * FL + r0] + threadIdx.x;
            UpGeo32 e[R];
            if (g0 < g_end)
            {
#pragma unroll
                for (int r = 0; r < R; r++)
                    e[r] = row[(size_t)r * ngroups + g0];
            }
            cp_async_wait_all();
            __syncthreads();
            for (int g = g0; g < g_end; g += blockDim.x)
            {
                if (g != g0)
                {
#pragma unroll
                    for (int r = 0; r < R; r++)
                        e[r] = row[(size_t)r * ngroups + g];
                }
                if (e[0].fe < 0)
                    continue;
                const int rl = e[0].pad - r0;
                if (rgf[r0 + rl] < 0)
                {
                    // tabulated element inactive in this child: absolute coordinates
                    const double xc[3] = {a.T.box_c[3 * box], a.T.box_c[3 * box + 1],
                                          a.T.box_c[3 * box + 2]};
#pragma unroll
                    for (int r = 0; r < R; r++)
                    {
                        if (e[r].node < 0)
                            continue;
                        double y[3];
                        node_position(a.G, el, e[r].node, a.hi_nodes, xc, a.T.box_H[box], y);
                        const double p[3] = {y[0] - a.T.box_c[3 * cb],
                                             y[1] - a.T.box_c[3 * cb + 1],
                                             y[2] - a.T.box_c[3 * cb + 2]};
                        float loc[3];
                        const int gf2 = fine_lookup_mixed(C, fm, p, a.T.box_H[cb], loc, a.err);
                        if (gf2 < 0)
                            continue;
                        const double e0 = y[0] - xc[0], e1 = y[1] - xc[1], e2 = y[2] - xc[2];
                        cplx<float> v = {0.f, 0.f};
                        cfmaf(v, ChebF<N0, N1, N2>::eval(fcf + (size_t)gf2 * P_LO, loc, a.lo),
                              transfer_mixed<KIND>(p[0] * p[0] + p[1] * p[1] + p[2] * p[2],
                                                   e0 * e0 + e1 * e1 + e2 * e2,
                                                   MK ? a.kp_plane[blockIdx.y] : a.kp));
                        acc[e[r].node].x += v.re;
                        acc[e[r].node].y += v.im;
                    }
                    continue;
                }
                float x[R][3], vr[R], vi[R];
#pragma unroll
                for (int r = 0; r < R; r++)
                    for (int d = 0; d < 3; d++)
                        x[r][d] = e[r].loc[d];
                ChebMulti<float, N0, N1, N2, R, true>::eval(blk + (size_t)rl * BS, x, a.lo, vr, vi);
                if constexpr (MK)
                {
#pragma unroll
                    for (int r = 0; r < R; r++)
                        if (e[r].node >= 0)
                        {
                            const cplx<float> t =
                                transfer_delta<KIND>(e[r].tr, e[r].ti, a.kp_plane[blockIdx.y]);
                            e[r].tr = t.re;
                            e[r].ti = t.im;
                        }
                }
#pragma unroll
                for (int r = 0; r < R; r++)
                    if (e[r].node >= 0)
                    {
                        const float2 s = acc[e[r].node];
                        acc[e[r].node] = make_float2(s.x + (vr[r] * e[r].tr - vi[r] * e[r].ti),
                                                     s.y + (vr[r] * e[r].ti + vi[r] * e[r].tr));
                    }
            }
        }
    }
    __syncthreads();
    float2* cv = reinterpret_cast<float2*>(a.cvals) + blockIdx.y * a.cv_plane;
    for (int n = threadIdx.x; n < a.P_hi; n += blockDim.x)
        cv[(size_t)c * a.P_hi + n] = acc[n];
}

} // namespace ifgf
#include "upward_tc.cuh"
namespace ifgf
{

template <int KIND, int N0, int N1, int N2>
__global__ void __launch_bounds__(UP_THREADS) upward_mixed_kernel(UpArgs a)
{
    constexpr int R = UPGEO_RUN;
    extern __shared__ float2 acc32[];
    const int c = a.idx[blockIdx.x];
    const int slot = a.slot[blockIdx.x];
    const int box = a.cc_box[c], el = a.cc_el[c];
    const float2* fcf = reinterpret_cast<const float2*>(a.fcoef);
    for (int n = threadIdx.x; n < a.P_hi; n += blockDim.x)
        acc32[n] = make_float2(0.f, 0.f);
    const LevelGeom& C = a.GC;
    const long long nf = (long long)C.nf[0] * C.nf[1] * C.nf[2];
    for (int o = 0; o < 8; o++)
    {
        const int cb = a.T.box_child[8 * box + o];
        if (cb < 0)
            continue;
        __syncthreads();
        const int* fm = a.fmap + C.fmap_off + (long long)(cb - C.box_off) * nf;
        const UpGeo32* row = a.geo32 + ((size_t)slot * 8 + o) * a.P_pad;
        const int ngroups = a.P_pad / R;
        for (int g = threadIdx.x; g < ngroups; g += blockDim.x)
        {
            UpGeo32 e[R];
#pragma unroll
            for (int r = 0; r < R; r++)
                e[r] = row[(size_t)r * ngroups + g];
            if (e[0].fe < 0)
                continue;
            const int gf = fm[e[0].fe];
            if (gf < 0)
            {
                // tabulated element inactive in this child: absolute coordinates
                const double xc[3] = {a.T.box_c[3 * box], a.T.box_c[3 * box + 1],
                                      a.T.box_c[3 * box + 2]};
#pragma unroll
                for (int r = 0; r < R; r++)
                {
                    if (e[r].node < 0)
                        continue;
                    double y[3];
                    node_position(a.G, el, e[r].node, a.hi_nodes, xc, a.T.box_H[box], y);
                    const double p[3] = {y[0] - a.T.box_c[3 * cb], y[1] - a.T.box_c[3 * cb + 1],
                                         y[2] - a.T.box_c[3 * cb + 2]};
                    float loc[3];
                    const int gf2 = fine_lookup_mixed(C, fm, p, a.T.box_H[cb], loc, a.err);
                    if (gf2 < 0)
                        continue;
                    const double e0 = y[0] - xc[0], e1 = y[1] - xc[1], e2 = y[2] - xc[2];
                    cplx<float> v = {0.f, 0.f};
                    cfmaf(v, ChebF<N0, N1, N2>::eval(fcf + (size_t)gf2 * a.P_lo, loc, a.lo),
                          transfer_mixed<KIND>(p[0] * p[0] + p[1] * p[1] + p[2] * p[2],
                                               e0 * e0 + e1 * e1 + e2 * e2, a.kp));
                    acc32[e[r].node].x += v.re;
                    acc32[e[r].node].y += v.im;
                }
                continue;
            }
            float x[R][3], vr[R], vi[R];
#pragma unroll
            for (int r = 0; r < R; r++)
                for (int d = 0; d < 3; d++)
                    x[r][d] = e[r].loc[d];
            ChebMulti<float, N0, N1, N2, R>::eval(fcf + (size_t)gf * a.P_lo, x, a.lo, vr, vi);
#pragma unroll
            for (int r = 0; r < R; r++)
                if (e[r].node >= 0)
                {
                    const float2 s = acc32[e[r].node];
                    acc32[e[r].node] = make_float2(s.x + (vr[r] * e[r].tr - vi[r] * e[r].ti),
                                                   s.y + (vr[r] * e[r].ti + vi[r] * e[r].tr));
                }
        }
    }
    __syncthreads();
    float2* cv = reinterpret_cast<float2*>(a.cvals);
    for (int n = threadIdx.x; n < a.P_hi; n += blockDim.x)
        cv[(size_t)c * a.P_hi + n] = acc32[n];
}


static __global__ void __launch_bounds__(256) coarse_to_fine_mixed_kernel(C2FArgs a)
{
    extern __shared__ float2 s2f[];
    const int c = a.idx ? a.idx[blockIdx.x] : (int)blockIdx.x;
    const int box = a.cc_box[c], el = a.cc_el[c];
    const int h0 = a.hi[0], h1 = a.hi[1], h2 = a.hi[2];
    const int F0 = a.f[0] * a.lo[0], F1 = a.f[1] * a.lo[1];
    const int sz0 = a.P_hi;
    const int sz2 = max(F0 * h1 * h2, F0 * F1 * a.lo[2]);
    float2* B0 = s2f;
    float2* B2 = B0 + sz0;
    float2* B1 = B2 + sz2;
    const double* A0 = a.A;
    const double* A1 = A0 + F0 * h0;
    const double* A2 = A1 + F1 * h1;
    const float2* cv = reinterpret_cast<const float2*>(a.cvals);
    float2* fco = reinterpret_cast<float2*>(a.fcoef);

    for (int i = threadIdx.x; i < sz0; i += blockDim.x)
        B0[i] = cv[(size_t)c * a.P_hi + i];
    __syncthreads();
    for (int o = threadIdx.x; o < F0 * h1 * h2; o += blockDim.x)
    {
        const int i0 = o % F0, r = o / F0;
        float re = 0, im = 0;
        for (int m = 0; m < h0; m++)
        {
            const float av = (float)A0[i0 * h0 + m];
            const float2 v = B0[m + h0 * r];
            re = fmaf(av, v.x, re);
            im = fmaf(av, v.y, im);
        }
        B2[o] = make_float2(re, im);
    }
    __syncthreads();
    for (int o = threadIdx.x; o < F0 * F1 * h2; o += blockDim.x)
    {
        const int i0 = o % F0, r = o / F0;
        const int i1 = r % F1, m2 = r / F1;
        float re = 0, im = 0;
        for (int m = 0; m < h1; m++)
        {
            const float av = (float)A1[i1 * h1 + m];
            const float2 v = B2[i0 + F0 * (m + h1 * m2)];
            re = fmaf(av, v.x, re);
            im = fmaf(av, v.y, im);
        }
        B1[o] = make_float2(re, im);
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
        for (int o = threadIdx.x; o < F0 * F1 * lo2; o += blockDim.x)
        {
            const int i01 = o % (F0 * F1), i2 = o / (F0 * F1);
            const int row = j2 * lo2 + i2;
            float re = 0, im = 0;
            for (int m = 0; m < h2; m++)
            {
                const float av = (float)A2[row * h2 + m];
                const float2 v = B1[i01 + F0 * F1 * m];
                re = fmaf(av, v.x, re);
                im = fmaf(av, v.y, im);
            }
            B2[o] = make_float2(re, im);
        }
        __syncthreads();
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
            fco[(size_t)gf * a.P_lo + q] = B2[(j0 * lo0 + i0) + F0 * ((j1 * lo1 + i1) + F1 * i2)];
        }
    }
}

// Coarse-to-fine with compile-time orders and refinement factor F (the same
// in every dimension), for the common order triples.  T is the working
// precision (double, or float in the mixed pipeline); the three matrices are
// staged in shared memory in T.
template <typename T> struct Vec2;
template <> struct Vec2<double>
{
    using type = double2;
};
template <> struct Vec2<float>
{
    using type = float2;
};

// The three per-dimension matrices as a kernel parameter: with every loop
// unrolled, each entry is a compile-time offset into the parameter bank and
// enters its FMA as a constant operand, so the contraction reads only the
// data operand from shared memory.
template <int H0, int H1, int H2, int L0, int L1, int L2, int F, typename T>
struct C2FMats
{
    T a0[F * L0 * H0];
    T a1[F * L1 * H1];
    T a2[F * L2 * H2];
};

// Row stride of the second intermediate: F0 F1 rounded up so that the rows
// of consecutive m2 start F0 banks apart (conflict-free stage-2 stores).
template <int F0, int F1>
__host__ __device__ constexpr int c2f_row_stride()
{
    int s = F0 * F1;
    while (s % 16 != F0 % 16)
        s++;
    return s;
}

// stage 2 of the fixed coarse-to-fine kernel: threads per fine column
// block j0 (its L0 x H2 row vectors, whole warps, so that a warp works for
// one j0 only)
template <int H2, int L0> __host__ __device__ constexpr int c2f_stage2_group()
{
    return (L0 * H2 + 31) / 32 * 32;
}

// one thread per row vector of the widest of the three stages
template <int H0, int H1, int H2, int L0, int L1, int L2, int F>
constexpr int c2f_fixed_threads()
{
    constexpr int s1 = H1 * H2, s2 = F * c2f_stage2_group<H2, L0>(), s3 = F * L0 * F * L1;
    constexpr int m = s1 > s2 ? (s1 > s3 ? s1 : s3) : (s2 > s3 ? s2 : s3);
    return (m + 31) / 32 * 32;
}

// Coarse-to-fine with compile-time orders and refinement factor F (the same
// in every dimension), one coarse cone per block, register-tiled: every
// thread loads one input vector of a mode product into registers once and
// produces all output rows that use it.
//   stage 1 (thread = (m1, m2)):  Y1[i0][m1][m2] = sum_m A0[i0][m] X[m][m1][m2]
//   stage 2 (thread = (i0, m2)):  Y2[m2][i0 + F0 i1] = sum_m A1[i1][m] Y1[i0][m][m2]
//   stage 3 (thread = i0 + F0 i1): C[j2 L2 + i2] = sum_m A2[j2 L2 + i2][m] Y2[m][.]
// Stage 3 writes the coefficients of every active sub-cone straight to
// global memory.  Warps follow the sub-cones: a stage-2 warp works for one
// fine column block j0 and skips the row blocks j1 whose sub-cones (j0, j1,
// j2) are all inactive; stage-3 threads go sub-cone by sub-cone (L0 L1 each),
// so that a warp spans about two sub-cones, skips the j2 where they are
// inactive and writes each active one's rows as contiguous runs.  NPL
// planes per CTA (blockIdx.y: planes NPL y ...): each matrix constant, index
// and barrier then serves NPL row vectors (2 for FP32 batches: 3.15 -> 3.03
// ms per batched matvec at N = 1e6).  T is the working precision (double,
// or float in the mixed pipeline).
template <int H0, int H1, int H2, int L0, int L1, int L2, int F, typename T, int NPL>
__global__ void __launch_bounds__(c2f_fixed_threads<H0, H1, H2, L0, L1, L2, F>())
    coarse_to_fine_fixed_kernel(C2FArgs a, const C2FMats<H0, H1, H2, L0, L1, L2, F, T> M)
{
    using V = typename Vec2<T>::type;
    constexpr int F0 = F * L0, F1 = F * L1;
    constexpr int P_HI = H0 * H1 * H2, P_LO = L0 * L1 * L2;
    constexpr int S2 = c2f_row_stride<F0, F1>();
    constexpr int Y1N = F0 * H1 * H2, YN = Y1N + S2 * H2; // elements per plane
    extern __shared__ __align__(16) unsigned char c2f_raw[];
    // plane p: Y1 at p YN ([m2][m1][i0], i0 fastest), Y2 at p YN + Y1N ([m2][S2])
    V* Y = reinterpret_cast<V*>(c2f_raw);
    __shared__ int gsub[F * F * F];
    const int c = a.idx ? a.idx[blockIdx.x] : (int)blockIdx.x;
    const int t = threadIdx.x;
    const int box = a.cc_box[c], el = a.cc_el[c];
    const int p0 = blockIdx.y * NPL; // first plane of the CTA
    if (t < F * F * F)
    {
        const int nc0 = a.G.nc[0], nc1 = a.G.nc[1];
        const int hid0 = el % nc0, hid1 = (el / nc0) % nc1, hid2 = el / (nc0 * nc1);
        const int nf0 = a.G.nf[0], nf1 = a.G.nf[1];
        const long long nft = (long long)nf0 * nf1 * a.G.nf[2];
        const int* fm = a.fmap + a.G.fmap_off + (long long)(box - a.G.box_off) * nft;
        const int j0 = t % F, j1 = (t / F) % F, j2 = t / (F * F);
        gsub[t] = fm[((hid2 * F + j2) * nf1 + (hid1 * F + j1)) * nf0 + (hid0 * F + j0)];
    }
    if (t < H1 * H2)
    {
        V x[NPL][H0];
#pragma unroll
        for (int p = 0; p < NPL; p++)
        {
            const V* src = reinterpret_cast<const V*>(a.cvals) + (p0 + p) * a.cv_plane +
                           (size_t)c * P_HI + H0 * t;
#pragma unroll
            for (int m = 0; m < H0; m++)
                x[p][m] = src[m];
        }
#pragma unroll
        for (int i0 = 0; i0 < F0; i0++)
        {
#pragma unroll
            for (int p = 0; p < NPL; p++)
            {
                T re = 0, im = 0;
#pragma unroll
                for (int m = 0; m < H0; m++)
                {
                    re = fma(M.a0[i0 * H0 + m], x[p][m].x, re);
                    im = fma(M.a0[i0 * H0 + m], x[p][m].y, im);
                }
                Y[p * YN + i0 + F0 * t] = V{re, im};
            }
        }
    }
    __syncthreads();
    constexpr int G2 = c2f_stage2_group<H2, L0>();
    if (t < F * G2 && t % G2 < L0 * H2)
    {
        const int j0 = t / G2, u = t % G2;
        const int i0 = j0 * L0 + u % L0, m2 = u / L0;
        V x[NPL][H1];
#pragma unroll
        for (int p = 0; p < NPL; p++)
#pragma unroll
            for (int m = 0; m < H1; m++)
                x[p][m] = Y[p * YN + i0 + F0 * (m + H1 * m2)];
#pragma unroll
        for (int j1 = 0; j1 < F; j1++)
        {
            bool used = false;
#pragma unroll
            for (int j2 = 0; j2 < F; j2++)
                used |= gsub[j0 + F * (j1 + F * j2)] >= 0;
            if (!used)
                continue; // no active sub-cone reads these rows
#pragma unroll
            for (int i1 = j1 * L1; i1 < (j1 + 1) * L1; i1++)
            {
#pragma unroll
                for (int p = 0; p < NPL; p++)
                {
                    T re = 0, im = 0;
#pragma unroll
                    for (int m = 0; m < H1; m++)
                    {
                        re = fma(M.a1[i1 * H1 + m], x[p][m].x, re);
                        im = fma(M.a1[i1 * H1 + m], x[p][m].y, im);
                    }
                    Y[p * YN + Y1N + i0 + F0 * i1 + S2 * m2] = V{re, im};
                }
            }
        }
    }
    __syncthreads();
    if (t < F0 * F1)
    {
        const int q = t % (L0 * L1), sc = t / (L0 * L1);
        const int i0 = q % L0, i1 = q / L0, j0 = sc % F, j1 = sc / F;
        const int i0f = j0 * L0 + i0, i1f = j1 * L1 + i1;
        V x[NPL][H2];
#pragma unroll
        for (int p = 0; p < NPL; p++)
#pragma unroll
            for (int m = 0; m < H2; m++)
                x[p][m] = Y[p * YN + Y1N + i0f + F0 * i1f + S2 * m];
#pragma unroll
        for (int j2 = 0; j2 < F; j2++)
        {
            const int gf = gsub[j0 + F * (j1 + F * j2)];
            if (gf < 0)
                continue;
#pragma unroll
            for (int i2 = 0; i2 < L2; i2++)
            {
#pragma unroll
                for (int p = 0; p < NPL; p++)
                {
                    T re = 0, im = 0;
#pragma unroll
                    for (int m = 0; m < H2; m++)
                    {
                        re = fma(M.a2[(j2 * L2 + i2) * H2 + m], x[p][m].x, re);
                        im = fma(M.a2[(j2 * L2 + i2) * H2 + m], x[p][m].y, im);
                    }
                    V* fco = reinterpret_cast<V*>(a.fcoef) + (p0 + p) * a.fc_plane;
                    fco[(size_t)gf * P_LO + i0 + L0 * i1 + L0 * L1 * i2] = V{re, im};
                }
            }
        }
    }
}

template <int H0, int H1, int H2, int L0, int L1, int L2, int F, typename T>
constexpr size_t c2f_fixed_smem(int npl = 1)
{
    constexpr int F0 = F * L0, F1 = F * L1;
    return (size_t)npl * (F0 * H1 * H2 + c2f_row_stride<F0, F1>() * H2) * 2 * sizeof(T);
}

// Launches the fixed-size coarse-to-fine kernel when (hi, lo, f) is one of the
// instantiated shapes; returns false otherwise.
template <typename T>
static bool launch_c2f_fixed(const C2FArgs& fa, const double* A_host, unsigned grid,
                             cudaStream_t st, unsigned planes = 1)
{
    const int* h = fa.hi;
    const int* l = fa.lo;
    const int f = fa.f[0];
    if (fa.f[1] != f || fa.f[2] != f || (f != 3 && f != 1) || A_host == nullptr)
        return false;
    // refinement factor 3 (fine grid 3x the coarse one) or 1 (the modified
    // Helmholtz kernel: fine = coarse grid)
#define IFGF_C2F_CASE_F(A, B, C, D, E, G, F)                                                  \
    {                                                                                          \
        C2FMats<A, B, C, D, E, G, F, T> mats;                                                  \
        T* dst = mats.a0;                                                                      \
        constexpr int NA = F * (D * A + E * B + G * C);                                        \
        static_assert(sizeof(mats) == NA * sizeof(T), "matrix block layout");                  \
        for (int i = 0; i < NA; i++)                                                           \
            dst[i] = (T)A_host[i];                                                             \
        /* FP32: two planes per CTA share every matrix constant and index */                  \
        constexpr int NPL = std::is_same<T, float>::value ? 2 : 1;                             \
        const int npl = planes % NPL == 0 ? NPL : 1;                                           \
        const size_t sm = c2f_fixed_smem<A, B, C, D, E, G, F, T>(npl);                         \
        auto kern = npl == 2 ? coarse_to_fine_fixed_kernel<A, B, C, D, E, G, F, T, NPL>        \
                             : coarse_to_fine_fixed_kernel<A, B, C, D, E, G, F, T, 1>;         \
        if (sm > 48 * 1024)                                                                    \
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);  \
        kern<<<dim3(grid, planes / npl), c2f_fixed_threads<A, B, C, D, E, G, F>(), sm, st>>>(  \
            fa, mats);                                                                         \
        return true;                                                                           \
    }
#define IFGF_C2F_CASE(A, B, C, D, E, G)                                                       \
    if (h[0] == A && h[1] == B && h[2] == C && l[0] == D && l[1] == E && l[2] == G)            \
    {                                                                                          \
        if (f == 3)                                                                            \
            IFGF_C2F_CASE_F(A, B, C, D, E, G, 3)                                               \
        else                                                                                   \
            IFGF_C2F_CASE_F(A, B, C, D, E, G, 1)                                               \
    }
    IFGF_C2F_CASE(5, 8, 8, 2, 5, 5)
    IFGF_C2F_CASE(6, 9, 9, 3, 6, 6)
    IFGF_C2F_CASE(7, 10, 10, 4, 7, 7)
#undef IFGF_C2F_CASE
#undef IFGF_C2F_CASE_F
    return false;
}

// Mixed-precision target leaf evaluation: near-field terms in FP32 on
// coordinates relative to the leaf's first target, far-field Chebyshev sums
// in FP32, every contribution accumulated in FP64.
template <int KIND, int N0, int N1, int N2, int PART>
__global__ void __launch_bounds__(PART == EVAL_FAR ? FAR_THREADS : EVAL_THREADS, PART == EVAL_FAR ? 3 : 6)
    target_eval_mixed_kernel(EvalArgs a)
{
    constexpr int TH = PART == EVAL_FAR ? FAR_THREADS : EVAL_THREADS;
    using P = PluginF<KIND>;
    // kernels with normals stage FP64 coordinates (see PluginF::kernel_d)
    using CT = typename std::conditional<P::needs_normals, double, float>::type;
    __shared__ CT xs[TH], ys[TH], zs[TH];
    __shared__ float wr[TH], wi[TH];
    __shared__ double n0[P::needs_normals ? TH : 1], n1[P::needs_normals ? TH : 1],
        n2[P::needs_normals ? TH : 1];
    __shared__ double rr[TH], ri[TH];
    constexpr int NF = PART == EVAL_FAR ? TH : 1;
    __shared__ double fcx[NF], fcy[NF], fcz[NF], fH[NF];
    __shared__ long long ffm[NF];
    __shared__ int flev[NF];
    __shared__ LookupF lfs[PART == EVAL_FAR ? MAX_LEVELS : 1];
    if (PART == EVAL_FAR)
        for (int l = threadIdx.x; l < a.L; l += blockDim.x)
            make_lookupf(a.lv[l], lfs[l]); // read after the first chunk's barriers
    const float2* wf = reinterpret_cast<const float2*>(a.w);
    const float2* fcf = reinterpret_cast<const float2*>(a.fcoef);
    const int tl = blockIdx.x;
    const int tf = a.tl_first[tl], tlast = a.tl_last[tl];
    const double r0 = a.tx[tf], r1 = a.ty[tf], r2 = a.tz[tf]; // local origin
    const long long nb0 = a.near_off[tl], nb1 = PART == EVAL_NEAR ? a.near_off[tl + 1] : nb0;
    const long long fb0 = a.far_off[tl], fb1 = PART == EVAL_FAR ? a.far_off[tl + 1] : fb0;
    for (int base = tf; base < tlast; base += TH)
    {
        const int cnt = min(TH, tlast - base);
        const int S = TH / cnt;
        const int ti = threadIdx.x % cnt, si = threadIdx.x / cnt;
        const bool active = si < S;
        const int t = base + ti;
        const double y0 = a.tx[t], y1 = a.ty[t], y2 = a.tz[t];
        const float yl0 = (float)(y0 - r0), yl1 = (float)(y1 - r1), yl2 = (float)(y2 - r2);
        double accr = 0, acci = 0;
        for (long long e = nb0; e < nb1; e++)
        {
            const int sb = a.near_src[e];
            const int sf = a.T.box_first[sb], sl = a.T.box_last[sb];
            for (int cs = sf; cs < sl; cs += TH)
            {
                const int ccnt = min(TH, sl - cs);
                __syncthreads();
                if (threadIdx.x < ccnt)
                {
                    const int i = cs + threadIdx.x;
                    xs[threadIdx.x] = (CT)(a.S.sx[i] - r0);
                    ys[threadIdx.x] = (CT)(a.S.sy[i] - r1);
                    zs[threadIdx.x] = (CT)(a.S.sz[i] - r2);
                    const float2 wv = wf[i];
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
                if (active)
                {
                    cplx<float> acc = {0.f, 0.f};
                    if constexpr (P::needs_normals)
                    {
                        const double yd0 = y0 - r0, yd1 = y1 - r1, yd2 = y2 - r2;
                        for (int i = si; i < ccnt; i += S)
                        {
                            const double x[3] = {xs[i] - yd0, ys[i] - yd1, zs[i] - yd2};
                            const double nv[3] = {n0[i], n1[i], n2[i]};
                            cfmaf(acc, cplx<float>{wr[i], wi[i]}, P::kernel_d(x, nv, a.kp));
                        }
                    }
                    else
                    {
                        for (int i = si; i < ccnt; i += S)
                        {
                            const float x[3] = {xs[i] - yl0, ys[i] - yl1, zs[i] - yl2};
                            cfmaf(acc, cplx<float>{wr[i], wi[i]}, P::kernel(x, nullptr, a.kp));
                        }
                    }
                    accr += acc.re;
                    acci += acc.im;
                }
            }
        }
        // far sources in chunks of TH boxes, whose centre, size,
        // level and fine-map row are staged in shared memory first
        for (long long e0 = fb0; e0 < fb1; e0 += TH)
        {
            const int fcnt = (int)min((long long)TH, fb1 - e0);
            __syncthreads();
            if (threadIdx.x < fcnt)
            {
                const int sb = a.far_src[e0 + threadIdx.x];
                const int lev = a.T.box_level[sb];
                const LevelGeom& G = a.lv[lev];
                const long long nft = (long long)G.nf[0] * G.nf[1] * G.nf[2];
                fcx[threadIdx.x] = a.T.box_c[3 * sb];
                fcy[threadIdx.x] = a.T.box_c[3 * sb + 1];
                fcz[threadIdx.x] = a.T.box_c[3 * sb + 2];
                fH[threadIdx.x] = a.T.box_H[sb];
                ffm[threadIdx.x] = G.fmap_off + (long long)(sb - G.box_off) * nft;
                flev[threadIdx.x] = lev;
            }
            __syncthreads();
            if (!active)
                continue;
            for (int i = si; i < fcnt; i += S)
            {
                const int lev = flev[i];
                const double p[3] = {y0 - fcx[i], y1 - fcy[i], y2 - fcz[i]};
                float loc[3];
                const int gf =
                    fine_lookup_fast(lfs[lev], a.lv[lev], a.fmap + ffm[i], p, fH[i], loc, a.err);
                if (gf < 0)
                    continue;
                const cplx<float> v = ChebF<N0, N1, N2>::eval(fcf + (size_t)gf * a.P_lo, loc, a.lo);
                const cplx<float> cf = cf_mixed<KIND>(p[0] * p[0] + p[1] * p[1] + p[2] * p[2], a.kp);
                accr += (double)(v.re * cf.re - v.im * cf.im);
                acci += (double)(v.re * cf.im + v.im * cf.re);
            }
        }
        __syncthreads();
        rr[threadIdx.x] = accr;
        ri[threadIdx.x] = acci;
        __syncthreads();
        if (active && si == 0)
        {
            double sr = 0, sim = 0;
            for (int s = 0; s < S; s++)
            {
                sr += rr[ti + s * cnt];
                sim += ri[ti + s * cnt];
            }
            if (PART == EVAL_NEAR)
                a.unear[t] = make_double2(sr, sim);
            else
            {
                const double2 nr = a.unear[t];
                sr += nr.x;
                sim += nr.y;
                const long long o = a.tgt_perm[t];
                if (a.real_out)
                    a.out[o] = sr;
                else
                {
                    a.out[2 * o] = sr;
                    a.out[2 * o + 1] = sim;
                }
            }
        }
    }
}

#define IFGF_CHECK(x)                                                                         \
    do                                                                                         \
    {                                                                                          \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess)                                                                 \
            throw Error(2, std::string(#x) + ": " + cudaGetErrorString(e_));                   \
    } while (0)

#define IFGF_CHECK_LAUNCH()                                                                   \
    do                                                                                         \
    {                                                                                          \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess)                                                                 \
            throw Error(2, std::string("kernel launch: ") + cudaGetErrorString(e_));          \
    } while (0)

// threads of a node CTA (NPT nodes per thread, a multiple of 32, at most
// NODE_THREADS) and the number of node chunks (grid.y) covering P_hi nodes
inline int node_threads(int P_hi)
{
    int t = (P_hi + NPT - 1) / NPT;
    t = (t + 31) / 32 * 32;
    return t < 32 ? 32 : (t > NODE_THREADS ? NODE_THREADS : t);
}
inline int node_chunks(int P_hi)
{
    const int per = NPT * node_threads(P_hi);
    return (P_hi + per - 1) / per;
}

#include "far_staged.cuh"

template <int KIND, int N0, int N1, int N2, bool MIXED>
static int run_mult(const MultPtrs& m, const void* d_w, void* d_u, bool real, cudaStream_t st,
                    LaunchHooks* hk)
{
    int launches = 0;
    const size_t c2f_smem = MIXED ? m.c2f_smem / 2 : m.c2f_smem;
    if (c2f_smem > 48 * 1024)
    {
        const cudaError_t e = MIXED ? cudaFuncSetAttribute(coarse_to_fine_mixed_kernel,
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                           (int)c2f_smem)
                                    : cudaFuncSetAttribute(coarse_to_fine_kernel,
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                           (int)c2f_smem);
        if (e != cudaSuccess)
            throw Error(2, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    }
    {
        const int thr = 256;
        const int blocks = (int)std::min<long long>((m.n_src + thr - 1) / thr, 148 * 16);
        if (hk)
            hk->begin(PROF_PERMUTE);
        if (MIXED)
            permute_weights_mixed_kernel<<<blocks, thr, 0, st>>>(
                (const double*)d_w, real ? 1 : 0, m.src_perm, reinterpret_cast<float2*>(m.w), m.n_src);
        else
            permute_weights_kernel<<<blocks, thr, 0, st>>>((const double*)d_w, real ? 1 : 0,
                                                           m.src_perm, m.w, m.n_src);
        IFGF_CHECK_LAUNCH();
        if (hk)
            hk->end();
        launches++;
    }
    // target evaluation arguments; the near pass needs only the permuted
    // densities, so without per-kernel timing it runs on the side stream
    // while the level loop builds the interpolants
    EvalArgs ea;
    ea.lv = m.lv_dev;
    ea.L = m.L;
    ea.T = m.T;
    ea.S = m.S;
    ea.tx = m.tx;
    ea.ty = m.ty;
    ea.tz = m.tz;
    ea.tgt_perm = m.tgt_perm;
    ea.tl_first = m.tl_first;
    ea.tl_last = m.tl_last;
    ea.far_off = m.tl_far_off;
    ea.far_src = m.tl_far_src;
    ea.near_off = m.tl_near_off;
    ea.near_src = m.tl_near_src;
    ea.w = m.w;
    ea.fmap = m.fmap;
    ea.fcoef = m.fcoef;
    ea.out = (double*)d_u;
    ea.unear = m.unear;
    ea.real_out = real ? 1 : 0;
    ea.err = m.err;
    ea.P_lo = m.P_lo;
    for (int d = 0; d < 3; d++)
        ea.lo[d] = m.lo[d];
    ea.kp = m.kp;
    const bool overlap = hk == nullptr && m.side != nullptr;
    if (m.n_tleaf > 0)
    {
        cudaStream_t ns = st;
        if (overlap)
        {
            IFGF_CHECK(cudaEventRecord(m.ev_fork, st));
            IFGF_CHECK(cudaStreamWaitEvent(m.side, m.ev_fork, 0));
            ns = m.side;
        }
        if (hk)
            hk->begin(PROF_NEAR);
        if (MIXED)
            target_eval_mixed_kernel<KIND, 0, 0, 0, EVAL_NEAR><<<m.n_tleaf, EVAL_THREADS, 0, ns>>>(ea);
        else
            target_eval_kernel<KIND, 0, 0, 0, EVAL_NEAR><<<m.n_tleaf, EVAL_THREADS, 0, ns>>>(ea);
        IFGF_CHECK_LAUNCH();
        if (hk)
            hk->end();
        if (overlap)
            IFGF_CHECK(cudaEventRecord(m.ev_join, m.side));
        launches++;
    }
    const int nthr = node_threads(m.P_hi);
    const int nchk = node_chunks(m.P_hi);
    for (int l = m.L - 1; l >= 0; l--)
    {
        const LevelGeom& G = m.lv_host[l];
        if (G.n_coarse == 0)
            continue;
        const LevelLists& LL = m.lists[l];
        if (LL.n_leaf > 0)
        {
            LeafArgs la{G, m.T, m.S, LL.cc_box, LL.cc_el, LL.leaf_idx, m.hi_nodes, m.w, m.cvals,
                        m.P_hi, m.kp};
            if (hk)
                hk->begin(PROF_COARSE, l);
            if (MIXED)
                leaf_sample_mixed_kernel<KIND>
                    <<<dim3(LL.n_leaf, nchk), nthr, 9 * nthr * sizeof(float), st>>>(la);
            else
                leaf_sample_kernel<KIND>
                    <<<dim3(LL.n_leaf, nchk), nthr, 8 * nthr * sizeof(double), st>>>(la);
            IFGF_CHECK_LAUNCH();
            if (hk)
                hk->end();
            launches++;
        }
        if (LL.n_up > 0)
        {
            UpArgs ua;
            ua.G = G;
            ua.GC = l + 1 < m.L ? m.lv_host[l + 1] : G;
            ua.T = m.T;
            ua.cc_box = LL.cc_box;
            ua.cc_el = LL.cc_el;
            ua.idx = LL.up_idx;
            ua.slot = LL.up_slot;
            ua.geo64 = LL.geo64;
            ua.geo32 = LL.geo32;
            ua.P_pad = LL.up_pad;
            ua.fe_list = LL.fe_list;
            ua.rch = 0;
            ua.cv_plane = ua.fc_plane = 0;
            ua.fe_pad = LL.fe_pad;
            ua.hi_nodes = m.hi_nodes;
            ua.fmap = m.fmap;
            ua.fcoef = m.fcoef;
            ua.cvals = m.cvals;
            ua.err = m.err;
            ua.P_hi = m.P_hi;
            ua.P_lo = m.P_lo;
            for (int d = 0; d < 3; d++)
                ua.lo[d] = m.lo[d];
            ua.kp = m.kp;
            if (hk)
                hk->begin(PROF_UPWARD, l);
            bool staged = false;
            if constexpr (MIXED)
            {
                ua.tc_tiles = LL.tc_tiles;
                ua.tc_img = LL.tc_img;
                ua.tc_img_off = LL.tc_img_off;
                ua.tc_status = m.tc_status;
                staged = launch_upward_tc<KIND, N0, N1, N2>(ua, LL.n_tc_tiles, LL.tc_fill,
                                                            m.up_path, st, 1,
                                                            m.up_choice ? m.up_choice[l] : -1);
            }
            if constexpr (MIXED && N0 > 0 && (N0 * N1 * N2) % 2 == 0)
                if (!staged)
            {
                ua.rch = upward_staged_rch<N0, N1, N2>(LL.fe_pad);
                const size_t sm = upward_staged_smem<N0, N1, N2>(m.P_hi, ua.rch, LL.fe_pad);
                if (LL.fe_pad > 0 && sm <= UP_STAGED_SMEM_MAX)
                {
                    auto kern = upward_staged_kernel<KIND, N0, N1, N2>;
                    if (sm > 48 * 1024)
                        IFGF_CHECK(cudaFuncSetAttribute(
                            kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                    kern<<<LL.n_up, UPS_THREADS, sm, st>>>(ua);
                    staged = true;
                }
            }
            if (staged)
            {
            }
            else if (MIXED)
                upward_mixed_kernel<KIND, N0, N1, N2>
                    <<<LL.n_up, UP_THREADS, m.P_hi * sizeof(float2), st>>>(ua);
            else
                upward_kernel<KIND, N0, N1, N2>
                    <<<LL.n_up, UP_THREADS, m.P_hi * sizeof(double2), st>>>(ua);
            IFGF_CHECK_LAUNCH();
            if (hk)
                hk->end();
            launches++;
        }
        // a sharded operator refines its own cones only (n_c2f >= 0)
        const unsigned c2f_grid = LL.n_c2f >= 0 ? (unsigned)LL.n_c2f : (unsigned)G.n_coarse;
        if (c2f_grid == 0)
            continue;
        C2FArgs fa;
        fa.G = G;
        fa.idx = LL.n_c2f >= 0 ? LL.c2f_idx : nullptr;
        fa.cv_plane = fa.fc_plane = 0;
        fa.cc_box = LL.cc_box;
        fa.cc_el = LL.cc_el;
        fa.cvals = m.cvals;
        fa.A = m.A;
        fa.fmap = m.fmap;
        fa.fcoef = m.fcoef;
        for (int d = 0; d < 3; d++)
        {
            fa.hi[d] = m.hi[d];
            fa.lo[d] = m.lo[d];
            fa.f[d] = m.fct[d];
        }
        fa.P_hi = m.P_hi;
        fa.P_lo = m.P_lo;
        if (hk)
            hk->begin(PROF_C2F, l);
        if (launch_c2f_fixed<typename std::conditional<MIXED, float, double>::type>(
                fa, m.A_host, c2f_grid, st))
        {
        }
        else if (MIXED)
            coarse_to_fine_mixed_kernel<<<c2f_grid, 256, c2f_smem, st>>>(fa);
        else
            coarse_to_fine_kernel<<<c2f_grid, 256, c2f_smem, st>>>(fa);
        IFGF_CHECK_LAUNCH();
        if (hk)
            hk->end();
        launches++;
    }
    if (m.n_tleaf > 0)
    {
        if (overlap)
            IFGF_CHECK(cudaStreamWaitEvent(st, m.ev_join, 0));
        if (hk)
            hk->begin(PROF_EVAL);
        if (MIXED)
            target_eval_mixed_kernel<KIND, N0, N1, N2, EVAL_FAR><<<m.n_tleaf, FAR_THREADS, 0, st>>>(ea);
        else
            target_eval_kernel<KIND, N0, N1, N2, EVAL_FAR><<<m.n_tleaf, EVAL_THREADS, 0, st>>>(ea);
        IFGF_CHECK_LAUNCH();
        if (hk)
            hk->end();
        launches++;
    }
    return launches;
}

template <int KIND>
int launch_mult_kernels(const MultPtrs& m, const void* d_w, void* d_u, bool real, cudaStream_t st,
                        LaunchHooks* hk)
{
    const int* lo = m.lo;
#define IFGF_RUN(A, B, C)                                                                     \
    return m.mixed ? run_mult<KIND, A, B, C, true>(m, d_w, d_u, real, st, hk)                  \
                   : run_mult<KIND, A, B, C, false>(m, d_w, d_u, real, st, hk)
    if (lo[0] == 2 && lo[1] == 5 && lo[2] == 5)
        IFGF_RUN(2, 5, 5);
    if (lo[0] == 3 && lo[1] == 6 && lo[2] == 6)
        IFGF_RUN(3, 6, 6);
    if (lo[0] == 4 && lo[1] == 7 && lo[2] == 7)
        IFGF_RUN(4, 7, 7);
    IFGF_RUN(0, 0, 0);
#undef IFGF_RUN
}

template <int KIND>
void permute_only(const MultPtrs& m, const void* d_w, bool real, cudaStream_t st)
{
    const int thr = 256;
    const int blocks = (int)std::min<long long>((m.n_src + thr - 1) / thr, 148 * 16);
    permute_weights_kernel<<<blocks, thr, 0, st>>>((const double*)d_w, real ? 1 : 0, m.src_perm,
                                                   m.w, m.n_src);
    IFGF_CHECK_LAUNCH();
}

template <int KIND>
void launch_direct_kernel(const MultPtrs& m, const int* tpos, int nt, double2* out, cudaStream_t st)
{
    direct_eval_kernel<KIND><<<nt, 256, 0, st>>>(m.S, m.w, m.n_src, m.tx, m.ty, m.tz, tpos, m.kp, out);
    IFGF_CHECK_LAUNCH();
}

// One thread per node, the sample box's sources read through L1: at most
// 10 samples of (order + 4)^3 nodes x leaf-size sources, once per estimate.
template <int KIND>
__global__ void __launch_bounds__(256) order_probe_kernel(ProbeArgs a)
{
    using P = Plugin<KIND>;
    const int s = blockIdx.y;
    const int n = a.node_off[s] + blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.node_off[s + 1])
        return;
    const double y[3] = {a.nodes[3 * n], a.nodes[3 * n + 1], a.nodes[3 * n + 2]};
    const double* xc = a.centre + 3 * s;
    const double e0 = y[0] - xc[0], e1 = y[1] - xc[1], e2 = y[2] - xc[2];
    const double dc = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
    cplx<double> acc = {0.0, 0.0};
    for (int i = a.src_off[s]; i < a.src_off[s + 1]; i++)
    {
        const double av[3] = {a.S.sx[i] - y[0], a.S.sy[i] - y[1], a.S.sz[i] - y[2]};
        const double nv[3] = {P::needs_normals ? a.S.nx[i] : 0.0,
                              P::needs_normals ? a.S.ny[i] : 0.0,
                              P::needs_normals ? a.S.nz[i] : 0.0};
        acc = cadd(acc, P::factored(av, nv, {1.0, 0.0}, y, dc, a.kp));
    }
    a.out[n] = make_double2(acc.re, acc.im);
}

template <int KIND>
void launch_order_probe(const ProbeArgs& a, int n_samples, int max_nodes, cudaStream_t st)
{
    if (n_samples <= 0 || max_nodes <= 0)
        return;
    order_probe_kernel<KIND><<<dim3((max_nodes + 255) / 256, n_samples), 256, 0, st>>>(a);
    IFGF_CHECK_LAUNCH();
}

#include "mult_batch.cuh"

#define IFGF_INSTANTIATE_KIND(K)                                                              \
    template int launch_mult_kernels<K>(const MultPtrs&, const void*, void*, bool, cudaStream_t, \
                                        LaunchHooks*);                                         \
    template int launch_mult_batch_kernels<K>(const MultPtrs&, const BatchPtrs&, const void*,  \
                                              void*, bool, cudaStream_t, LaunchHooks*);        \
    template int tune_upward_kernels<K>(const MultPtrs&, const BatchPtrs*, int, cudaStream_t,   \
                                        signed char*, double*, double*);                       \
    template void launch_direct_kernel<K>(const MultPtrs&, const int*, int, double2*, cudaStream_t); \
    template void permute_only<K>(const MultPtrs&, const void*, bool, cudaStream_t);         \
    template void launch_order_probe<K>(const ProbeArgs&, int, int, cudaStream_t);             \
    template void launch_build_upgeo<K>(const LevelGeom&, const LevelGeom&, double, double,   \
                                        const double*, const int*, int, const double*, int,     \
                                        KParams, int, UpGeo64*, UpGeo32*, int, int2*);          \
    template int upgeo_row_max<K>(const LevelGeom&, const LevelGeom&, double, double,         \
                                  const double*, const int*, int, const double*, int, KParams,  \
                                  int*, int*, int*);

} // namespace ifgf
