// Mixed-precision matvec of several right-hand sides at once (included by
// mult_kernels.cuh).  The BATCH_NB densities of a plane group share every
// geometry- and kernel-dependent quantity of the pipeline -- the
// factored-kernel values at the cone nodes, the near-field kernel values, the
// far-field cone lookups and centred factors -- and keep their own
// interpolant planes (plane p at offset p * plane of each buffer).  One
// launch per stage and level covers all groups (a grid dimension selects the
// group).  The upward transfer and the coarse-to-fine step run the
// single-right-hand-side kernels with blockIdx.y selecting the plane.
// Multi-wavenumber batches (MK): every plane has its own wavenumber
// (BatchPtrs::kp_plane); the planes then share the geometry only -- node and
// source positions, cone lookups, Chebyshev bases -- and evaluate their
// kernel values, centred and centre-shift factors each.
// Included inside namespace ifgf, after the single-right-hand-side kernels.
#pragma once


// Permuted FP32 densities of nrhs right-hand sides; planes past nrhs zero.
static __global__ void permute_batch_kernel(const double* __restrict__ in, int real_in,
                                            const long long* __restrict__ perm, float2* w,
                                            long long n, int nrhs, long long in_plane)
{
    const int b = blockIdx.y;
    float2* wb = w + (size_t)b * n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
    {
        if (b >= nrhs)
        {
            wb[i] = make_float2(0.f, 0.f);
            continue;
        }
        const long long j = perm[i];
        const double* src = in + (size_t)b * in_plane;
        if (real_in)
            wb[i] = make_float2((float)src[j], 0.f);
        else
        {
            const double2 v = reinterpret_cast<const double2*>(src)[j];
            wb[i] = make_float2((float)v.x, (float)v.y);
        }
    }
}

// Leaf sampling of a plane group (blockIdx.z): the factored kernel at a
// (node, source) pair is evaluated once with unit density and applied to
// every plane's density (the kernels are linear in the density); with MK once
// per plane, at its wavenumber.  Each thread takes LEAF_NPT nodes, and a
// source's data (relative position and squared distance as one float4, the
// planes' densities as two) are read from shared memory once for all of
// them (measured per batched matvec at N = 1e6, p = 9: 2 nodes 3.23 ms, 3
// nodes 3.17, 4 nodes 3.06, 6 nodes 3.88).
constexpr int LEAF_NPT = 4;
// with MK every (node, plane) pair has its own kernel evaluation, so more
// nodes per thread save no evaluations: two, at fewer registers (the
// 64-wavenumber CQ batch at N = 1e5: 61.8 ms, 66.6 with four)
__host__ __device__ constexpr int leaf_npt(bool mk) { return mk ? 2 : LEAF_NPT; }
inline int leaf_batch_threads(int P_hi, int npt)
{
    int t = (P_hi + npt - 1) / npt;
    t = (t + 31) / 32 * 32;
    return t < 32 ? 32 : (t > NODE_THREADS ? NODE_THREADS : t);
}
inline int leaf_batch_chunks(int P_hi, int npt)
{
    const int per = npt * leaf_batch_threads(P_hi, npt);
    return (P_hi + per - 1) / per;
}
// dynamic shared memory: per source slot a float4, BATCH_NB float2 and the
// normal's three floats
inline size_t leaf_batch_smem(int nt)
{
    return (size_t)nt * (sizeof(float4) + BATCH_NB * sizeof(float2) + 3 * sizeof(float));
}

template <int KIND, bool MK>
__global__ void __launch_bounds__(NODE_THREADS) leaf_sample_batch_kernel(LeafArgs a, BatchPtrs bp)
{
    using P = PluginF<KIND>;
    constexpr int NB = BATCH_NB, NPQ = leaf_npt(MK);
    static_assert(NB % 2 == 0, "the planes' densities are read as float4 pairs");
    extern __shared__ __align__(16) float4 leaf_sm4[];
    __shared__ KParams kps[MK ? NB : 1];
    const int pb = blockIdx.z * NB; // first plane of the group
    if constexpr (MK)
        if (threadIdx.x < NB)
            kps[threadIdx.x] = bp.kp_plane[pb + threadIdx.x]; // read after the chunk barriers
    const int c = a.idx[blockIdx.x];
    const int node0 = blockIdx.y * NPQ * blockDim.x;
    const int box = a.cc_box[c], el = a.cc_el[c];
    const double xc[3] = {a.T.box_c[3 * box], a.T.box_c[3 * box + 1], a.T.box_c[3 * box + 2]};
    const double H = a.T.box_H[box];
    float b[NPQ][3], dc[NPQ];
    bool live[NPQ];
    cplx<float> acc[NPQ][NB];
#pragma unroll
    for (int q = 0; q < NPQ; q++)
    {
        const int n = node0 + threadIdx.x + q * blockDim.x;
#pragma unroll
        for (int r = 0; r < NB; r++)
            acc[q][r] = {0.f, 0.f};
        b[q][0] = b[q][1] = b[q][2] = 0.f;
        dc[q] = 1.f;
        live[q] = n < a.P_hi;
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
    float4* sa = leaf_sm4;                                 // [nt] (x, y, z, |.|^2)
    float4* sw = sa + nt;                                  // [nt][NB / 2] densities
    float* n0 = reinterpret_cast<float*>(sw + nt * NB / 2); // [nt] x 3 normals
    float* n1 = n0 + nt;
    float* n2 = n1 + nt;
    const int f = a.T.box_first[box], l = a.T.box_last[box];
    for (int cs = f; cs < l; cs += nt)
    {
        const int cnt = min(nt, l - cs);
        __syncthreads();
        if (threadIdx.x < cnt)
        {
            const int i = cs + threadIdx.x;
            const double a0 = a.S.sx[i] - xc[0], a1 = a.S.sy[i] - xc[1], a2 = a.S.sz[i] - xc[2];
            sa[threadIdx.x] =
                make_float4((float)a0, (float)a1, (float)a2, (float)(a0 * a0 + a1 * a1 + a2 * a2));
#pragma unroll
            for (int r = 0; r < NB; r += 2)
            {
                const float2 u = bp.w[(size_t)(pb + r) * bp.n_src + i];
                const float2 v = bp.w[(size_t)(pb + r + 1) * bp.n_src + i];
                sw[threadIdx.x * (NB / 2) + r / 2] = make_float4(u.x, u.y, v.x, v.y);
            }
            if (P::needs_normals)
            {
                n0[threadIdx.x] = (float)a.S.nx[i];
                n1[threadIdx.x] = (float)a.S.ny[i];
                n2[threadIdx.x] = (float)a.S.nz[i];
            }
        }
        __syncthreads();
        // sources outer, nodes inner: each source's data is read from shared
        // memory once for all of the thread's nodes (every node's sum still
        // runs over the sources in order)
        for (int i = 0; i < cnt; i++)
        {
            const float4 s4 = sa[i];
            const float av[3] = {s4.x, s4.y, s4.z};
            const float aai = s4.w;
            const float nv[3] = {P::needs_normals ? n0[i] : 0.f, P::needs_normals ? n1[i] : 0.f,
                                 P::needs_normals ? n2[i] : 0.f};
            float2 wr[NB];
#pragma unroll
            for (int r = 0; r < NB; r += 2)
            {
                const float4 u = sw[i * (NB / 2) + r / 2];
                wr[r] = make_float2(u.x, u.y);
                wr[r + 1] = make_float2(u.z, u.w);
            }
#pragma unroll
            for (int q = 0; q < NPQ; q++)
            {
                if (!live[q])
                    continue;
                if constexpr (MK)
                {
#pragma unroll
                    for (int r = 0; r < NB; r++)
                    {
                        const cplx<float> v =
                            P::factored(av, aai, b[q], nv, {1.f, 0.f}, dc[q], kps[r]);
                        acc[q][r].re = fmaf(wr[r].x, v.re, fmaf(-wr[r].y, v.im, acc[q][r].re));
                        acc[q][r].im = fmaf(wr[r].x, v.im, fmaf(wr[r].y, v.re, acc[q][r].im));
                    }
                }
                else
                {
                    const cplx<float> v = P::factored(av, aai, b[q], nv, {1.f, 0.f}, dc[q], a.kp);
#pragma unroll
                    for (int r = 0; r < NB; r++)
                    {
                        acc[q][r].re = fmaf(wr[r].x, v.re, fmaf(-wr[r].y, v.im, acc[q][r].re));
                        acc[q][r].im = fmaf(wr[r].x, v.im, fmaf(wr[r].y, v.re, acc[q][r].im));
                    }
                }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NPQ; q++)
    {
        const int n = node0 + threadIdx.x + q * blockDim.x;
        if (n < a.P_hi)
#pragma unroll
            for (int r = 0; r < NB; r++)
                bp.cvals[(size_t)(pb + r) * bp.cv_plane + (size_t)c * a.P_hi + n] =
                    make_float2(acc[q][r].re, acc[q][r].im);
    }
}

// Near field of a plane group (blockIdx.y): one kernel value per (target,
// source) pair, applied to every plane (with MK one per plane); FP32 per
// source chunk, FP64 across chunks and threads, written to the near-sum
// planes.
template <int KIND, bool MK>
__global__ void __launch_bounds__(EVAL_THREADS) near_batch_kernel(EvalArgs a, BatchPtrs bp)
{
    using P = PluginF<KIND>;
    constexpr int NB = BATCH_NB;
    __shared__ KParams kps[MK ? NB : 1];
    const int pb = blockIdx.y * NB;
    if constexpr (MK)
        if (threadIdx.x < NB)
            kps[threadIdx.x] = bp.kp_plane[pb + threadIdx.x]; // read after the chunk barriers
    using CT = typename std::conditional<P::needs_normals, double, float>::type;
    __shared__ CT xs[EVAL_THREADS], ys[EVAL_THREADS], zs[EVAL_THREADS];
    __shared__ float2 ws[NB][EVAL_THREADS];
    __shared__ double n0[P::needs_normals ? EVAL_THREADS : 1], n1[P::needs_normals ? EVAL_THREADS : 1],
        n2[P::needs_normals ? EVAL_THREADS : 1];
    __shared__ double rr[NB][EVAL_THREADS], ri[NB][EVAL_THREADS];
    const long long nsrc = bp.n_src;
    const int tl = blockIdx.x;
    const int tf = a.tl_first[tl], tlast = a.tl_last[tl];
    const double r0 = a.tx[tf], r1 = a.ty[tf], r2 = a.tz[tf];
    const long long nb0 = a.near_off[tl], nb1 = a.near_off[tl + 1];
    for (int base = tf; base < tlast; base += EVAL_THREADS)
    {
        const int cnt = min(EVAL_THREADS, tlast - base);
        const int S = EVAL_THREADS / cnt;
        const int ti = threadIdx.x % cnt, si = threadIdx.x / cnt;
        const bool active = si < S;
        const int t = base + ti;
        const double y0 = a.tx[t], y1 = a.ty[t], y2 = a.tz[t];
        const float yl0 = (float)(y0 - r0), yl1 = (float)(y1 - r1), yl2 = (float)(y2 - r2);
        double accr[NB], acci[NB];
#pragma unroll
        for (int r = 0; r < NB; r++)
            accr[r] = acci[r] = 0.0;
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
                    xs[threadIdx.x] = (CT)(a.S.sx[i] - r0);
                    ys[threadIdx.x] = (CT)(a.S.sy[i] - r1);
                    zs[threadIdx.x] = (CT)(a.S.sz[i] - r2);
#pragma unroll
                    for (int r = 0; r < NB; r++)
                        ws[r][threadIdx.x] = bp.w[(size_t)(pb + r) * nsrc + i];
                    if (P::needs_normals)
                    {
                        n0[threadIdx.x] = a.S.nx[i];
                        n1[threadIdx.x] = a.S.ny[i];
                        n2[threadIdx.x] = a.S.nz[i];
                    }
                }
                __syncthreads();
                if (!active)
                    continue;
                cplx<float> acc[NB];
#pragma unroll
                for (int r = 0; r < NB; r++)
                    acc[r] = {0.f, 0.f};
                for (int i = si; i < ccnt; i += S)
                {
                    if constexpr (P::needs_normals)
                    {
                        const double yd0 = y0 - r0, yd1 = y1 - r1, yd2 = y2 - r2;
                        const double x[3] = {xs[i] - yd0, ys[i] - yd1, zs[i] - yd2};
                        const double nv[3] = {n0[i], n1[i], n2[i]};
                        if constexpr (MK)
                        {
#pragma unroll
                            for (int r = 0; r < NB; r++)
                                cfmaf(acc[r], cplx<float>{ws[r][i].x, ws[r][i].y},
                                      P::kernel_d(x, nv, kps[r]));
                        }
                        else
                        {
                            const cplx<float> kv = P::kernel_d(x, nv, a.kp);
#pragma unroll
                            for (int r = 0; r < NB; r++)
                                cfmaf(acc[r], cplx<float>{ws[r][i].x, ws[r][i].y}, kv);
                        }
                    }
                    else
                    {
                        const float x[3] = {xs[i] - yl0, ys[i] - yl1, zs[i] - yl2};
                        if constexpr (MK)
                        {
#pragma unroll
                            for (int r = 0; r < NB; r++)
                                cfmaf(acc[r], cplx<float>{ws[r][i].x, ws[r][i].y},
                                      P::kernel(x, nullptr, kps[r]));
                        }
                        else
                        {
                            const cplx<float> kv = P::kernel(x, nullptr, a.kp);
#pragma unroll
                            for (int r = 0; r < NB; r++)
                                cfmaf(acc[r], cplx<float>{ws[r][i].x, ws[r][i].y}, kv);
                        }
                    }
                }
#pragma unroll
                for (int r = 0; r < NB; r++)
                {
                    accr[r] += acc[r].re;
                    acci[r] += acc[r].im;
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < NB; r++)
        {
            rr[r][threadIdx.x] = accr[r];
            ri[r][threadIdx.x] = acci[r];
        }
        __syncthreads();
        if (active && si == 0)
        {
#pragma unroll
            for (int r = 0; r < NB; r++)
            {
                double sr = 0, sim = 0;
                for (int s = 0; s < S; s++)
                {
                    sr += rr[r][ti + s * cnt];
                    sim += ri[r][ti + s * cnt];
                }
                bp.unear[(size_t)(pb + r) * bp.n_tgt + t] = make_double2(sr, sim);
            }
        }
    }
}

// Enqueues the batched mixed matvec of bp.nrhs (<= bp.groups * BATCH_NB)
// right-hand sides, one launch per stage and level; returns the number of
// kernels launched, or -1 when this operator's shape has no batched path
// (runtime orders, or a level whose upward runs do not fit the staged kernel)
// and the right-hand sides must run one by one.
template <int KIND, int N0, int N1, int N2, bool MK>
static int run_mult_batch(const MultPtrs& m, const BatchPtrs& bp, const void* d_w, void* d_u,
                          bool real, cudaStream_t st, LaunchHooks* hk)
{
    if constexpr (N0 == 0 || (N0 * N1 * N2) % 2 != 0)
        return -1;
    else
    {
        for (int l = 0; l + 1 < m.L; l++)
        {
            const LevelLists& LL = m.lists[l];
            if (LL.n_up > 0 && (LL.fe_pad <= 0 || upward_staged_smem<N0, N1, N2>(
                                                      m.P_hi,
                                                      upward_staged_rch<N0, N1, N2>(LL.fe_pad),
                                                      LL.fe_pad) >
                                                      UP_STAGED_SMEM_MAX))
                return -1;
        }
        if (m.lo[0] != N0 || m.fct[1] != m.fct[0] || m.fct[2] != m.fct[0] ||
            (m.fct[0] != 3 && m.fct[0] != 1))
            return -1;
        int launches = 0;
        {
            const int thr = 256;
            const int blocks = (int)std::min<long long>((m.n_src + thr - 1) / thr, 148 * 4);
            if (hk)
                hk->begin(PROF_PERMUTE);
            permute_batch_kernel<<<dim3(blocks, bp.groups * BATCH_NB), thr, 0, st>>>(
                (const double*)d_w, real ? 1 : 0, m.src_perm, bp.w, m.n_src, bp.nrhs, bp.in_plane);
            IFGF_CHECK_LAUNCH();
            if (hk)
                hk->end();
            launches++;
        }
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
        ea.w = reinterpret_cast<const double2*>(bp.w);
        ea.fmap = m.fmap;
        ea.fcoef = reinterpret_cast<const double2*>(bp.fcoef);
        ea.out = (double*)d_u;
        ea.unear = bp.unear;
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
            near_batch_kernel<KIND, MK><<<dim3(m.n_tleaf, bp.groups), EVAL_THREADS, 0, ns>>>(ea, bp);
            IFGF_CHECK_LAUNCH();
            if (hk)
                hk->end();
            if (overlap)
                IFGF_CHECK(cudaEventRecord(m.ev_join, m.side));
            launches++;
        }
        const int nthr = leaf_batch_threads(m.P_hi, leaf_npt(MK));
        const int nchk = leaf_batch_chunks(m.P_hi, leaf_npt(MK));
        for (int l = m.L - 1; l >= 0; l--)
        {
            const LevelGeom& G = m.lv_host[l];
            if (G.n_coarse == 0)
                continue;
            const LevelLists& LL = m.lists[l];
            if (LL.n_leaf > 0)
            {
                LeafArgs la{G,      m.T,     m.S,  LL.cc_box, LL.cc_el, LL.leaf_idx, m.hi_nodes,
                            m.w,    m.cvals, m.P_hi, m.kp};
                if (hk)
                    hk->begin(PROF_COARSE, l);
                leaf_sample_batch_kernel<KIND, MK>
                    <<<dim3(LL.n_leaf, nchk, bp.groups), nthr, leaf_batch_smem(nthr), st>>>(la, bp);
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
                ua.geo32 = MK ? bp.dgeo32[l] : LL.geo32;
                ua.P_pad = LL.up_pad;
                ua.fe_list = LL.fe_list;
                ua.fe_pad = LL.fe_pad;
                ua.rch = upward_staged_rch<N0, N1, N2>(LL.fe_pad);
                ua.kp_plane = bp.kp_plane;
                ua.cv_plane = bp.cv_plane;
                ua.fc_plane = bp.fc_plane;
                ua.hi_nodes = m.hi_nodes;
                ua.fmap = m.fmap;
                ua.fcoef = reinterpret_cast<const double2*>(bp.fcoef);
                ua.cvals = reinterpret_cast<double2*>(bp.cvals);
                ua.err = m.err;
                ua.P_hi = m.P_hi;
                ua.P_lo = m.P_lo;
                for (int d = 0; d < 3; d++)
                    ua.lo[d] = m.lo[d];
                ua.kp = m.kp;
                if (hk)
                    hk->begin(PROF_UPWARD, l);
                bool tensor = false;
                if (!MK && bp.tc_tiles)
                {
                    ua.tc_tiles = bp.tc_tiles[l];
                    ua.tc_img = LL.tc_img;
                    ua.tc_img_off = LL.tc_img_off;
                    ua.tc_status = m.tc_status;
                    tensor = launch_upward_tc<KIND, N0, N1, N2>(
                        ua, bp.n_tc_tiles[l], bp.tc_fill[l], m.up_path, st, bp.groups * BATCH_NB,
                        bp.up_choice ? bp.up_choice[l] : -1);
                }
                if (!tensor)
                {
                    const size_t sm = upward_staged_smem<N0, N1, N2>(m.P_hi, ua.rch, LL.fe_pad);
                    auto kern = upward_staged_kernel<KIND, N0, N1, N2, MK>;
                    if (sm > 48 * 1024)
                        IFGF_CHECK(cudaFuncSetAttribute(
                            kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                    kern<<<dim3(LL.n_up, bp.groups * BATCH_NB), UPS_THREADS, sm, st>>>(ua);
                }
                IFGF_CHECK_LAUNCH();
                if (hk)
                    hk->end();
                launches++;
            }
            const unsigned c2f_grid = LL.n_c2f >= 0 ? (unsigned)LL.n_c2f : (unsigned)G.n_coarse;
            if (c2f_grid == 0)
                continue;
            C2FArgs fa;
            fa.G = G;
            fa.idx = LL.n_c2f >= 0 ? LL.c2f_idx : nullptr;
            fa.cv_plane = bp.cv_plane;
            fa.fc_plane = bp.fc_plane;
            fa.cc_box = LL.cc_box;
            fa.cc_el = LL.cc_el;
            fa.cvals = reinterpret_cast<const double2*>(bp.cvals);
            fa.A = m.A;
            fa.fmap = m.fmap;
            fa.fcoef = reinterpret_cast<double2*>(bp.fcoef);
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
            if (!launch_c2f_fixed<float>(fa, m.A_host, c2f_grid, st, bp.groups * BATCH_NB))
                throw Error(6, "batched coarse-to-fine needs one of the fixed order shapes");
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
            if (bp.fp_chunk)
            {
                auto launch_plan = [&](auto nsl) {
                    constexpr int NSL = decltype(nsl)::value;
                    constexpr size_t fsm = far_plan_smem<N0 * N1 * N2, BATCH_NB, NSL>();
                    auto fk = far_plan_kernel<KIND, N0, N1, N2, MK, BATCH_NB, NSL>;
                    IFGF_CHECK(cudaFuncSetAttribute(
                        fk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm));
                    fk<<<dim3(bp.fp_nchunk, bp.groups), FARB_THREADS, fsm, st>>>(ea, bp);
                    return cudaSuccess;
                };
                if (bp.fp_nslot <= FAR_PLAN_SLOTS_FEW)
                    IFGF_CHECK(launch_plan(std::integral_constant<int, FAR_PLAN_SLOTS_FEW>{}));
                else if (bp.fp_nslot <= FAR_PLAN_SLOTS_MID)
                    IFGF_CHECK(launch_plan(std::integral_constant<int, FAR_PLAN_SLOTS_MID>{}));
                else
                    IFGF_CHECK(launch_plan(std::integral_constant<int, FAR_PLAN_SLOTS>{}));
            }
            else
            {
                constexpr size_t fsm = far_batch_smem<N0, N1, N2, BATCH_NB>();
                auto fk = far_batch_kernel<KIND, N0, N1, N2, MK, BATCH_NB>;
                IFGF_CHECK(cudaFuncSetAttribute(fk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                (int)fsm));
                fk<<<dim3(m.n_tleaf, bp.groups), FARB_THREADS, fsm, st>>>(ea, bp);
            }
            IFGF_CHECK_LAUNCH();
            if (hk)
                hk->end();
            launches++;
        }
        return launches;
    }
}

// The upward-kernel autotuner of one order shape (see tune_upward_kernels).
template <int KIND, int N0, int N1, int N2>
static int tune_upward_shape(const MultPtrs& m, const BatchPtrs* bp, int planes, cudaStream_t st,
                             signed char* choice, double* ms_ffma, double* ms_tc)
{
    for (int l = 0; l < m.L; l++)
    {
        choice[l] = -1;
        ms_ffma[l] = ms_tc[l] = 0;
    }
    if constexpr (!uptc_shape<N0, N1, N2>())
        return 0;
    else
    {
        cudaEvent_t e0, e1;
        IFGF_CHECK(cudaEventCreate(&e0));
        IFGF_CHECK(cudaEventCreate(&e1));
        struct Ev
        {
            cudaEvent_t a, b;
            ~Ev()
            {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
            }
        } ev{e0, e1};
        auto timed = [&](auto&& launch) {
            float best = 1e30f;
            for (int rep = 0; rep < 3; rep++)
            {
                IFGF_CHECK(cudaEventRecord(e0, st));
                launch();
                IFGF_CHECK_LAUNCH();
                IFGF_CHECK(cudaEventRecord(e1, st));
                IFGF_CHECK(cudaEventSynchronize(e1));
                float ms = 0;
                IFGF_CHECK(cudaEventElapsedTime(&ms, e0, e1));
                if (rep > 0 && ms < best) // the first launch warms up
                    best = ms;
            }
            return (double)best;
        };
        int tuned = 0;
        for (int l = 0; l + 1 < m.L; l++)
        {
            const LevelLists& LL = m.lists[l];
            const int4* tiles = bp ? bp->tc_tiles[l] : LL.tc_tiles;
            const int nt = bp ? bp->n_tc_tiles[l] : LL.n_tc_tiles;
            if (LL.n_up <= 0 || LL.fe_pad <= 0 || !tiles || nt <= 0)
                continue;
            UpArgs ua;
            ua.G = m.lv_host[l];
            ua.GC = m.lv_host[l + 1];
            ua.T = m.T;
            ua.cc_box = LL.cc_box;
            ua.cc_el = LL.cc_el;
            ua.idx = LL.up_idx;
            ua.slot = LL.up_slot;
            ua.geo64 = LL.geo64;
            ua.geo32 = LL.geo32;
            ua.P_pad = LL.up_pad;
            ua.fe_list = LL.fe_list;
            ua.fe_pad = LL.fe_pad;
            ua.rch = upward_staged_rch<N0, N1, N2>(LL.fe_pad);
            ua.cv_plane = bp ? bp->cv_plane : 0;
            ua.fc_plane = bp ? bp->fc_plane : 0;
            ua.hi_nodes = m.hi_nodes;
            ua.fmap = m.fmap;
            ua.fcoef = bp ? reinterpret_cast<const double2*>(bp->fcoef) : m.fcoef;
            ua.cvals = bp ? reinterpret_cast<double2*>(bp->cvals) : m.cvals;
            ua.err = m.err;
            ua.P_hi = m.P_hi;
            ua.P_lo = m.P_lo;
            for (int d = 0; d < 3; d++)
                ua.lo[d] = m.lo[d];
            ua.kp = m.kp;
            ua.tc_tiles = tiles;
            ua.tc_img = LL.tc_img;
            ua.tc_img_off = LL.tc_img_off;
            ua.tc_status = m.tc_status;
            const size_t sm = upward_staged_smem<N0, N1, N2>(m.P_hi, ua.rch, LL.fe_pad);
            if (sm > UP_STAGED_SMEM_MAX ||
                uptc_smem_bytes<N0, N1, N2>(m.P_hi, LL.fe_pad) > 227 * 1024)
                continue;
            auto kern = upward_staged_kernel<KIND, N0, N1, N2, false>;
            if (sm > 48 * 1024)
                IFGF_CHECK(
                    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            ms_ffma[l] = timed([&] { kern<<<dim3(LL.n_up, planes), UPS_THREADS, sm, st>>>(ua); });
            ms_tc[l] = timed([&] {
                launch_upward_tc<KIND, N0, N1, N2>(ua, nt, 1.f, UP_TENSOR, st, planes, 1);
            });
            choice[l] = ms_tc[l] < 0.97 * ms_ffma[l] ? 1 : 0;
            tuned++;
        }
        return tuned;
    }
}

template <int KIND>
int tune_upward_kernels(const MultPtrs& m, const BatchPtrs* bp, int planes, cudaStream_t st,
                        signed char* choice, double* ms_ffma, double* ms_tc)
{
    const int* lo = m.lo;
    if (lo[0] == 2 && lo[1] == 5 && lo[2] == 5)
        return tune_upward_shape<KIND, 2, 5, 5>(m, bp, planes, st, choice, ms_ffma, ms_tc);
    if (lo[0] == 3 && lo[1] == 6 && lo[2] == 6)
        return tune_upward_shape<KIND, 3, 6, 6>(m, bp, planes, st, choice, ms_ffma, ms_tc);
    for (int l = 0; l < m.L; l++)
    {
        choice[l] = -1;
        ms_ffma[l] = ms_tc[l] = 0;
    }
    return 0;
}

template <int KIND>
int launch_mult_batch_kernels(const MultPtrs& m, const BatchPtrs& bp, const void* d_w, void* d_u,
                              bool real, cudaStream_t st, LaunchHooks* hk)
{
    const int* lo = m.lo;
#define IFGF_RUN_BATCH(A, B, C)                                                               \
    return bp.kp_plane ? run_mult_batch<KIND, A, B, C, true>(m, bp, d_w, d_u, real, st, hk)     \
                       : run_mult_batch<KIND, A, B, C, false>(m, bp, d_w, d_u, real, st, hk)
    if (lo[0] == 2 && lo[1] == 5 && lo[2] == 5)
        IFGF_RUN_BATCH(2, 5, 5);
    if (lo[0] == 3 && lo[1] == 6 && lo[2] == 6)
        IFGF_RUN_BATCH(3, 6, 6);
    if (lo[0] == 4 && lo[1] == 7 && lo[2] == 7)
        IFGF_RUN_BATCH(4, 7, 7);
#undef IFGF_RUN_BATCH
    return -1;
}
