// Far-field evaluation with coefficient blocks staged in shared memory, for
// the batched mixed pipeline (NP = BATCH_NB planes per CTA).  A single plane
// does not pay for the staging (the per-box work is a quarter, the hashing,
// copies and barriers are not): the single right-hand-side pipeline keeps its
// direct kernel.  Included by mult_kernels.cuh inside namespace ifgf, after
// the evaluation helpers.
#pragma once

// Far field of a plane group (blockIdx.y; NP planes) for one target leaf per
// CTA (evaluateFromInterp, ifgfoperator.hpp:1736-1891, for every far source
// box of the leaf and of its ancestors).  Adds the near sums and writes the
// caller's result planes (the first nrhs).
//
// Thread (ti, si) owns target ti and far boxes si, si + S, ... (S = threads /
// targets): it looks up the fine cone of its (target, box) pair once for all
// NP planes, computes the centred factor and adds the pair's NP values to
// its FP64 sums.  For every S consecutive far boxes (one pair per thread):
//   1. the distinct cones of the pairs go into a small hash table; the first
//      far_slots() of them get a shared-memory slot for their NP-plane
//      coefficient blocks (cp.async copies);
//   2. the pairs are written as records (local coordinates, slot) in slot
//      order, each slot's group padded to 8 positions;
//   3. an evaluating thread takes positions 2q and 2q + 1 -- two pairs of
//      one cone -- for half of the planes, so every 16-byte coefficient load
//      feeds both pairs' FMAs, and the 4 lanes of a quad read one block (an
//      LDS.128 is then served in its minimum of one wavefront per
//      half-warp); the plane halves keep all threads busy;
//   4. the owner of each pair reads the pair's values back, applies the
//      factor and adds them, in box order.
// Evaluated in owner order, one pair per thread, the lanes of a warp read the
// few cones of their targets from unrelated slots: the shared loads split
// into about three wavefronts each, and with one pair per load the L1 data
// pipe, not the FMA pipe, bounds the kernel.  Pairs whose cone found no slot
// are sorted last, one per evaluating thread, and read global memory.
constexpr int FARB_THREADS = 256; // threads of one CTA (one pair each per group)
constexpr int FARB_CTAS = 2;      // resident CTAs per SM (registers: 128 per thread)
constexpr int FAR_HASH = 128;
constexpr int FAR_BOXES = 128; // far boxes whose geometry is loaded at once
constexpr int FAR_PAD = 8;     // positions per quad of evaluating lanes
template <int P_LO, int NP> __host__ __device__ constexpr int far_slot_stride()
{
    int s = NP * P_LO; // float2 per slot: NP planes, then pad to 16 B mod 128
    while ((s * 8) % 128 != 16 && (s * 8) % 128 != 80)
        s++;
    return s;
}
// record positions of one group of boxes: one pair per thread, plus the
// padding of each slot's group (at most FAR_PAD - 1 each)
__host__ __device__ constexpr int far_positions(int nslot)
{
    return (FARB_THREADS + (FAR_PAD - 1) * nslot + 7) / 8 * 8;
}
// static shared memory of far_batch_kernel, for the slot budget
template <int NP> __host__ __device__ constexpr int far_static_bytes(int nslot)
{
    return 3 * 2 * FAR_HASH * 4 + 2 * nslot * 4 + 16 + far_positions(nslot) * (16 + 8 * NP) +
           NP * (int)sizeof(KParams) + FAR_BOXES * (4 * 8 + 8 + 4) +
           MAX_LEVELS * (int)sizeof(LookupF);
}
// slots: as many as fit beside the static arrays with FARB_CTAS CTAs per SM
// (233472 bytes of shared memory per SM, 1 KB reserved per CTA, 512 bytes
// margin), at most 96 / NP (well inside the FAR_HASH entries) and 32 (one
// warp scans the slot counts)
template <int P_LO, int NP> __host__ __device__ constexpr int far_slots()
{
    int n = 96 / NP < 32 ? 96 / NP : 32;
    while (n > 1 && n * far_slot_stride<P_LO, NP>() * 8 + far_static_bytes<NP>(n) >
                        233472 / FARB_CTAS - 1024 - 512)
        n--;
    return n;
}
template <int N0, int N1, int N2, int NP> constexpr size_t far_batch_smem()
{
    constexpr size_t slots =
        (size_t)far_slots<N0 * N1 * N2, NP>() * far_slot_stride<N0 * N1 * N2, NP>() * 8;
    constexpr size_t red = 2 * NP * FARB_THREADS * sizeof(double); // final reduction
    return slots > red ? slots : red;
}
// record of a pair in slot order: local coordinates (float bits) and the slot,
// or ~(global fine cone) for a pair read from global memory
struct __align__(16) FarRec
{
    int l0, l1, l2, code;
};

// Two points of one cone block in shared memory: the tensor-product
// Chebyshev sums of ChebF, sharing every coefficient load.
template <int N0, int N1, int N2> struct ChebF2
{
    __device__ static __forceinline__ void basis(const float* x, float (&t0)[N0], float (&t1)[N1],
                                                 float (&t2)[N2])
    {
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
    }
    __device__ static __forceinline__ void eval(const float2* __restrict__ c, const float* xa,
                                                const float* xb, cplx<float>& va, cplx<float>& vb)
    {
        float a0[N0], a1[N1], a2[N2], b0[N0], b1[N1], b2[N2];
        basis(xa, a0, a1, a2);
        basis(xb, b0, b1, b2);
        // T_0 = 1: every sum starts from its first term instead of adding
        // it to zero (the same values; one instruction less per sum)
        float aar, aai, bar, bai;
#pragma unroll
        for (int k = 0; k < N2; k++)
        {
            float abr, abi, bbr, bbi;
#pragma unroll
            for (int j = 0; j < N1; j += CoefRows<N0, N1>::ROWS)
            {
                float2 v[CoefRows<N0, N1>::ROWS * N0];
                CoefRows<N0, N1, true>::load(c + N0 * (j + N1 * k), v);
#pragma unroll
                for (int jj = 0; jj < CoefRows<N0, N1>::ROWS; jj++)
                {
                    float acr = v[jj * N0].x, aci = v[jj * N0].y;
                    float bcr = acr, bci = aci;
#pragma unroll
                    for (int i = 1; i < N0; i++)
                    {
                        acr = fmaf(v[jj * N0 + i].x, a0[i], acr);
                        aci = fmaf(v[jj * N0 + i].y, a0[i], aci);
                        bcr = fmaf(v[jj * N0 + i].x, b0[i], bcr);
                        bci = fmaf(v[jj * N0 + i].y, b0[i], bci);
                    }
                    if (j + jj == 0)
                    {
                        abr = acr, abi = aci, bbr = bcr, bbi = bci;
                    }
                    else
                    {
                        abr = fmaf(acr, a1[j + jj], abr);
                        abi = fmaf(aci, a1[j + jj], abi);
                        bbr = fmaf(bcr, b1[j + jj], bbr);
                        bbi = fmaf(bci, b1[j + jj], bbi);
                    }
                }
            }
            if (k == 0)
            {
                aar = abr, aai = abi, bar = bbr, bai = bbi;
            }
            else
            {
                aar = fmaf(abr, a2[k], aar);
                aai = fmaf(abi, a2[k], aai);
                bar = fmaf(bbr, b2[k], bar);
                bai = fmaf(bbi, b2[k], bai);
            }
        }
        va = {aar, aai};
        vb = {bar, bai};
    }
};

template <int KIND, int N0, int N1, int N2, bool MK, int NP>
__global__ void __launch_bounds__(FARB_THREADS, FARB_CTAS)
    far_batch_kernel(EvalArgs a, BatchPtrs bp)
{
    constexpr int NB = NP;
    constexpr int P_LO = N0 * N1 * N2;
    constexpr int SS = far_slot_stride<P_LO, NP>();
    constexpr int NSLOT = far_slots<P_LO, NP>();
    constexpr int NPOS = far_positions(NSLOT);
    constexpr int CPP = P_LO / 2; // 16-byte chunks of one plane's block
    static_assert(P_LO % 2 == 0, "blocks must be whole 16-byte chunks");
    static_assert(NSLOT > 0, "one slot must fit");
    static_assert(NSLOT <= 32, "one warp scans the slot counts");
    extern __shared__ __align__(16) float2 far_sh[]; // slots; the final reduction reuses it
    __shared__ int hkey[2][FAR_HASH], hslot[2][FAR_HASH], hcnt[2][FAR_HASH];
    __shared__ int sgf[NSLOT], sent[NSLOT], nslot[2], novf[2];
    __shared__ FarRec frec[NPOS];
    __shared__ float2 fres[NB][NPOS];
    __shared__ KParams kps[MK ? NB : 1];
    const int pb = blockIdx.y * NB;
    if constexpr (MK)
        if (threadIdx.x < NB)
            kps[threadIdx.x] = bp.kp_plane[pb + threadIdx.x]; // read after the chunk barriers
    for (int q = threadIdx.x; q < 2 * FAR_HASH; q += blockDim.x)
    {
        hkey[q / FAR_HASH][q % FAR_HASH] = -1;
        hcnt[q / FAR_HASH][q % FAR_HASH] = 0;
    }
    if (threadIdx.x < 2)
        nslot[threadIdx.x] = novf[threadIdx.x] = 0;
    const int lane = threadIdx.x & 31;
    __shared__ double fcx[FAR_BOXES], fcy[FAR_BOXES], fcz[FAR_BOXES], fH[FAR_BOXES];
    __shared__ long long ffm[FAR_BOXES];
    __shared__ int flev[FAR_BOXES];
    __shared__ LookupF lfs[MAX_LEVELS];
    for (int l = threadIdx.x; l < a.L; l += blockDim.x)
        make_lookupf(a.lv[l], lfs[l]); // read after the first chunk's barriers
    const int tl = blockIdx.x;
    const int tf = a.tl_first[tl], tlast = a.tl_last[tl];
    const long long fb0 = a.far_off[tl], fb1 = a.far_off[tl + 1];
    int tab = 0; // hash table of the current group of boxes (CTA-uniform)
    for (int base = tf; base < tlast; base += FARB_THREADS)
    {
        const int cnt = min(FARB_THREADS, tlast - base);
        const int S = FARB_THREADS / cnt;
        const int ti = threadIdx.x % cnt, si = threadIdx.x / cnt;
        const bool active = si < S;
        const int t = base + ti;
        const double y0 = a.tx[t], y1 = a.ty[t], y2 = a.tz[t];
        double accr[NB], acci[NB];
#pragma unroll
        for (int r = 0; r < NB; r++)
            accr[r] = acci[r] = 0.0;
        for (long long e0 = fb0; e0 < fb1; e0 += FAR_BOXES)
        {
            const int fcnt = (int)min((long long)FAR_BOXES, fb1 - e0);
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
            // the cone of this thread's pair in box i of the chunk (g < 0: none)
            auto lookup = [&](int i, int& g, float (&l)[3], double& dd) {
                g = -1;
                l[0] = l[1] = l[2] = 0.f;
                dd = 0.0;
                if (active && i < fcnt)
                {
                    const int lev = flev[i];
                    const double p[3] = {y0 - fcx[i], y1 - fcy[i], y2 - fcz[i]};
                    g = fine_lookup_fast(lfs[lev], a.lv[lev], a.fmap + ffm[i], p, fH[i], l, a.err);
                    dd = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
                }
            };
            int gf_next;
            float loc_next[3];
            double d2_next;
            lookup(si, gf_next, loc_next, d2_next);
            // groups of S boxes: at most one pair per thread; every thread
            // runs every group (barriers inside).  The next group's lookup (a
            // dependent global load) is issued before this one's copies are
            // waited for.
            for (int c0 = 0; c0 < fcnt; c0 += S)
            {
                const int gf = gf_next;
                const float loc[3] = {loc_next[0], loc_next[1], loc_next[2]};
                const double d2 = d2_next;
                int h = -1, rank = 0;
                if (gf >= 0)
                {
                    // insert the cone, bounded linear probing; the first
                    // inserter takes a slot while slots last.  rank: this
                    // pair's place among the pairs of its cone.
                    int hh = (int)(((unsigned)gf * 2654435761u) >> 25) & (FAR_HASH - 1);
                    for (int q = 0; q < FAR_HASH; q++, hh = (hh + 1) & (FAR_HASH - 1))
                    {
                        const int prev = atomicCAS(&hkey[tab][hh], -1, gf);
                        if (prev == -1)
                        {
                            const int k = atomicAdd(&nslot[tab], 1);
                            if (k < NSLOT)
                            {
                                sgf[k] = gf;
                                sent[k] = hh;
                            }
                            hslot[tab][hh] = k < NSLOT ? k : -1;
                            h = hh;
                            break;
                        }
                        if (prev == gf)
                        {
                            h = hh;
                            break;
                        }
                    }
                    if (h >= 0)
                        rank = atomicAdd(&hcnt[tab][h], 1);
                }
                __syncthreads(); // table, slot list and counts complete
                const int ns = min(nslot[tab], NSLOT);
                // group starts: every warp scans the padded slot counts
                const int ck = lane < ns ? hcnt[tab][sent[lane]] : 0;
                const int pk = (ck + FAR_PAD - 1) & ~(FAR_PAD - 1);
                int incl = pk;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1)
                {
                    const int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o)
                        incl += v;
                }
                const int slotted = __shfl_sync(0xffffffffu, incl, 31); // padded
                const int k = h >= 0 ? hslot[tab][h] : -1;
                const int src = k >= 0 ? k : 0;
                const int kbase = __shfl_sync(0xffffffffu, incl - pk, src);
                const int kcnt = __shfl_sync(0xffffffffu, ck, src);
                const int kend = __shfl_sync(0xffffffffu, incl, src);
                int pos = -1;
                if (gf >= 0)
                {
                    pos = k >= 0 ? kbase + rank : slotted + atomicAdd(&novf[tab], 1);
                    frec[pos] = FarRec{__float_as_int(loc[0]), __float_as_int(loc[1]),
                                       __float_as_int(loc[2]), k >= 0 ? k : ~gf};
                    // the last pair of a slot fills its group's padding
                    // (coordinates 0: evaluated, never read)
                    if (k >= 0 && rank == kcnt - 1)
                        for (int p = kbase + kcnt; p < kend; p++)
                            frec[p] = FarRec{0, 0, 0, k};
                }
                // the other table was last read before this barrier: clear it
                for (int q = threadIdx.x; q < FAR_HASH; q += blockDim.x)
                {
                    hkey[tab ^ 1][q] = -1;
                    hcnt[tab ^ 1][q] = 0;
                }
                if (threadIdx.x == 0)
                    nslot[tab ^ 1] = novf[tab ^ 1] = 0;
                // one warp per slot, lanes over the slot's 16-byte chunks
                for (int ks = threadIdx.x >> 5; ks < ns; ks += FARB_THREADS / 32)
                {
                    const float2* src0 = bp.fcoef + (size_t)pb * bp.fc_plane + (size_t)sgf[ks] * P_LO;
                    float2* dst0 = far_sh + (size_t)ks * SS;
#pragma unroll
                    for (int r = 0; r < NB; r++)
                        for (int ch = lane; ch < CPP; ch += 32)
                            cp_async16(dst0 + r * P_LO + 2 * ch,
                                       src0 + (size_t)r * bp.fc_plane + 2 * ch);
                }
                lookup(c0 + S + si, gf_next, loc_next, d2_next);
                cp_async_wait_all();
                __syncthreads(); // blocks staged, records written
                // evaluate: work item = (two pairs of one slot, half of the
                // planes), then (one pair read from global memory, half of
                // the planes); consecutive threads take consecutive pairs
                constexpr int NH = NB > 1 ? 2 : 1, RH = NB / NH;
                static_assert(NB % NH == 0, "plane halves");
                const int n_two = slotted / 2, n_one = novf[tab];
                const int n_item = NH * (n_two + n_one);
                for (int w = threadIdx.x; w < n_item; w += FARB_THREADS)
                {
                    if (w < NH * n_two)
                    {
                        const int q = w % n_two, r0 = (w / n_two) * RH;
                        const FarRec ra = frec[2 * q], rb = frec[2 * q + 1];
                        const float la[3] = {__int_as_float(ra.l0), __int_as_float(ra.l1),
                                             __int_as_float(ra.l2)};
                        const float lb[3] = {__int_as_float(rb.l0), __int_as_float(rb.l1),
                                             __int_as_float(rb.l2)};
#pragma unroll
                        for (int rr = 0; rr < RH; rr++)
                        {
                            cplx<float> va, vb;
                            ChebF2<N0, N1, N2>::eval(far_sh + (size_t)ra.code * SS +
                                                         (r0 + rr) * P_LO,
                                                     la, lb, va, vb);
                            fres[r0 + rr][2 * q] = make_float2(va.re, va.im);
                            fres[r0 + rr][2 * q + 1] = make_float2(vb.re, vb.im);
                        }
                    }
                    else
                    {
                        const int w1 = w - NH * n_two;
                        const int p = slotted + w1 % n_one, r0 = (w1 / n_one) * RH;
                        const FarRec rc = frec[p];
                        const float l3[3] = {__int_as_float(rc.l0), __int_as_float(rc.l1),
                                             __int_as_float(rc.l2)};
#pragma unroll
                        for (int rr = 0; rr < RH; rr++)
                        {
                            const cplx<float> v = ChebF<N0, N1, N2>::eval(
                                bp.fcoef + (size_t)(pb + r0 + rr) * bp.fc_plane +
                                    (size_t)(~rc.code) * P_LO,
                                l3, a.lo);
                            fres[r0 + rr][p] = make_float2(v.re, v.im);
                        }
                    }
                }
                __syncthreads(); // values of every pair written
                if (gf >= 0)
                {
                    cplx<float> cf;
                    if constexpr (!MK)
                        cf = cf_mixed<KIND>(d2, a.kp);
#pragma unroll
                    for (int r = 0; r < NB; r++)
                    {
                        if constexpr (MK)
                            cf = cf_mixed<KIND>(d2, kps[r]);
                        const float2 v = fres[r][pos];
                        accr[r] += (double)(v.x * cf.re - v.y * cf.im);
                        acci[r] += (double)(v.x * cf.im + v.y * cf.re);
                    }
                }
                tab ^= 1;
            }
        }
        __syncthreads(); // the slots are no longer read: reduce through them
        double* rr = reinterpret_cast<double*>(far_sh);
        double* ri = rr + NB * FARB_THREADS;
#pragma unroll
        for (int r = 0; r < NB; r++)
        {
            rr[r * FARB_THREADS + threadIdx.x] = accr[r];
            ri[r * FARB_THREADS + threadIdx.x] = acci[r];
        }
        __syncthreads();
        if (active && si == 0)
        {
            const long long o = a.tgt_perm[t];
            for (int r = 0; r < NB && pb + r < bp.nrhs; r++)
            {
                double sr = 0, sim = 0;
                for (int s = 0; s < S; s++)
                {
                    sr += rr[r * FARB_THREADS + ti + s * cnt];
                    sim += ri[r * FARB_THREADS + ti + s * cnt];
                }
                const double2 nr = bp.unear[(size_t)(pb + r) * bp.n_tgt + t];
                sr += nr.x;
                sim += nr.y;
                double* out = a.out + (size_t)(pb + r) * bp.out_plane;
                if (a.real_out)
                    out[o] = sr;
                else
                {
                    out[2 * o] = sr;
                    out[2 * o + 1] = sim;
                }
            }
        }
    }
}

// The far field of far_batch_kernel from the far-field plan built at init
// (FarChunk / FarGroup / FarPlanRec): the cone lookups, the slot assignment
// and the cone-ordered, padded records of every group are read instead of
// computed, so a group is: copy its records and slot blocks (cp.async), the
// owners' box distances meanwhile, one barrier, the sums (two pairs of one
// slot per work item, as in far_batch_kernel), one barrier, the owners'
// factors and FP64 sums in box order, overlapping the next group's copies.
// (Prefetching the next group's blocks and records into L2 during this
// group's copies measured slower.)  One CTA per chunk of up to 256 targets of
// a leaf and per group of NP planes.
static_assert(FAR_PLAN_THREADS == FARB_THREADS && FAR_PLAN_PAD % 2 == 0,
              "the plan's owners are threads of 256, its work items pairs of one slot");
template <int P_LO, int NP, int NSL> __host__ __device__ constexpr size_t far_plan_smem()
{
    const size_t slots = (size_t)NSL * far_slot_stride<P_LO, NP>() * 8;
    const size_t red = 2 * NP * FARB_THREADS * sizeof(double); // final reduction
    return slots > red ? slots : red;
}

template <int KIND, int N0, int N1, int N2, bool MK, int NP, int NSL>
__global__ void __launch_bounds__(FARB_THREADS, far_plan_ctas(NSL, N0 * N1 * N2, NP))
    far_plan_kernel(EvalArgs a, BatchPtrs bp)
{
    constexpr int NB = NP;
    constexpr int P_LO = N0 * N1 * N2;
    constexpr int SS = far_slot_stride<P_LO, NP>();
    constexpr int CPP = P_LO / 2; // 16-byte chunks of one plane's block
    constexpr int NH = NB > 1 ? 2 : 1, RH = NB / NH;
    static_assert(NB % NH == 0, "plane halves");
    static_assert(FARB_THREADS == 256, "the plan's owner index is a thread of 256");
    extern __shared__ __align__(16) float2 far_sh[]; // slots; the final reduction reuses it
    __shared__ FarPlanRec frec[far_plan_pos(NSL)];
    __shared__ float2 fres[NB][FARB_THREADS + 1]; // column FARB_THREADS: padding
    __shared__ KParams kps[MK ? NB : 1];
    const int pb = blockIdx.y * NB;
    if constexpr (MK)
        if (threadIdx.x < NB)
            kps[threadIdx.x] = bp.kp_plane[pb + threadIdx.x]; // read after the first barrier
    const int lane = threadIdx.x & 31;
    const FarChunk C = bp.fp_chunk[blockIdx.x];
    const int cnt = C.cnt;
    const int S = FARB_THREADS / cnt;
    const int ti = threadIdx.x % cnt, si = threadIdx.x / cnt;
    const bool active = si < S;
    const int t = C.t0 + ti;
    const double y0 = a.tx[t], y1 = a.ty[t], y2 = a.tz[t];
    double accr[NB], acci[NB];
#pragma unroll
    for (int r = 0; r < NB; r++)
        accr[r] = acci[r] = 0.0;
    for (long long g = C.g0; g < C.g1; g++)
    {
        const FarGroup G = bp.fp_group[g];
        for (int i = threadIdx.x; i < G.npos; i += FARB_THREADS)
            cp_async16(&frec[i], bp.fp_rec + G.rec + i);
        // one warp per slot, lanes over the slot's 16-byte chunks
        for (int ks = threadIdx.x >> 5; ks < G.nslot; ks += FARB_THREADS / 32)
        {
            const int cone = bp.fp_slot[G.slot + ks];
            const float2* src0 = bp.fcoef + (size_t)pb * bp.fc_plane + (size_t)cone * P_LO;
            float2* dst0 = far_sh + (size_t)ks * SS;
#pragma unroll
            for (int r = 0; r < NB; r++)
                for (int ch = lane; ch < CPP; ch += 32)
                    cp_async16(dst0 + r * P_LO + 2 * ch, src0 + (size_t)r * bp.fc_plane + 2 * ch);
        }
        // this thread's pair: its box's distance, and a zero value in case
        // the pair has no record (no cone)
        const bool mine = active && si < G.nbox;
        double d2 = 0.0;
        if (mine)
        {
            const int sb = a.far_src[G.box0 + si];
            const double p0 = y0 - a.T.box_c[3 * sb], p1 = y1 - a.T.box_c[3 * sb + 1],
                         p2 = y2 - a.T.box_c[3 * sb + 2];
            d2 = p0 * p0 + p1 * p1 + p2 * p2;
        }
#pragma unroll
        for (int r = 0; r < NB; r++)
            fres[r][threadIdx.x] = make_float2(0.f, 0.f);
        cp_async_wait_all();
        __syncthreads(); // records and blocks staged
        const int n_two = G.nslotted / 2, n_one = G.npos - G.nslotted;
        // work item = (two pairs of one slot, or one pair from global
        // memory) x NHX of the planes: a group whose items would spill into
        // a second round of the threads takes smaller ones if the rounds
        // then cost less (rounds x planes per item, with 10 % for the bases
        // and records each item repeats)
        auto items = [&](auto nh) {
            constexpr int NHX = decltype(nh)::value, RHX = NB / NHX;
            const int n_item = NHX * (n_two + n_one);
            // item w = h n_two + q (two pairs 2q, 2q + 1, planes from h RHX),
            // then the one-pair items; q and h follow w without divisions
            int w = threadIdx.x, q = w, h = 0;
            while (h < NHX && q >= n_two)
                q -= n_two, h++;
            for (; h < NHX; w += FARB_THREADS)
            {
                const int r0 = h * RHX;
                const FarPlanRec ra = frec[2 * q], rb = frec[2 * q + 1];
                const float la[3] = {__int_as_float(ra.l0), __int_as_float(ra.l1),
                                     __int_as_float(ra.l2)};
                const float lb[3] = {__int_as_float(rb.l0), __int_as_float(rb.l1),
                                     __int_as_float(rb.l2)};
                const int k = (ra.w >> 9) & 31;
                const int oa = min(ra.w & 511, FARB_THREADS), ob = min(rb.w & 511, FARB_THREADS);
#pragma unroll
                for (int rr = 0; rr < RHX; rr++)
                {
                    cplx<float> va, vb;
                    ChebF2<N0, N1, N2>::eval(far_sh + (size_t)k * SS + (r0 + rr) * P_LO, la, lb,
                                             va, vb);
                    fres[r0 + rr][oa] = make_float2(va.re, va.im);
                    fres[r0 + rr][ob] = make_float2(vb.re, vb.im);
                }
                q += FARB_THREADS;
                while (h < NHX && q >= n_two)
                    q -= n_two, h++;
            }
            for (; w < n_item; w += FARB_THREADS)
            {
                const int w1 = w - NHX * n_two;
                const int j = w1 % n_one, r0 = (w1 / n_one) * RHX;
                const FarPlanRec rc = frec[G.nslotted + j];
                const float l3[3] = {__int_as_float(rc.l0), __int_as_float(rc.l1),
                                     __int_as_float(rc.l2)};
                const int cone = bp.fp_slot[G.slot + G.nslot + j];
                const int o = min(rc.w & 511, FARB_THREADS);
#pragma unroll
                for (int rr = 0; rr < RHX; rr++)
                {
                    const cplx<float> v = ChebF<N0, N1, N2>::eval(
                        bp.fcoef + (size_t)(pb + r0 + rr) * bp.fc_plane + (size_t)cone * P_LO, l3,
                        a.lo);
                    fres[r0 + rr][o] = make_float2(v.re, v.im);
                }
            }
        };
        const int n = n_two + n_one;
        const int rounds_h = (NH * n + FARB_THREADS - 1) / FARB_THREADS;
        const int rounds_q = (NB * n + FARB_THREADS - 1) / FARB_THREADS;
        if (NB > NH && 11 * rounds_q * (NB / NB) < 10 * rounds_h * (NB / NH))
            items(std::integral_constant<int, NB>{});
        else
            items(std::integral_constant<int, NH>{});
        __syncthreads(); // values of every pair written
        if (mine)
        {
            cplx<float> cf;
            if constexpr (!MK)
                cf = cf_mixed<KIND>(d2, a.kp);
#pragma unroll
            for (int r = 0; r < NB; r++)
            {
                if constexpr (MK)
                    cf = cf_mixed<KIND>(d2, kps[r]);
                const float2 v = fres[r][threadIdx.x];
                accr[r] += (double)(v.x * cf.re - v.y * cf.im);
                acci[r] += (double)(v.x * cf.im + v.y * cf.re);
            }
        }
        // no barrier: records and slots are not read after the last one, so
        // the next group's copies overlap these sums, and each thread zeroes
        // only its own value column
    }
    __syncthreads();
    double* rr = reinterpret_cast<double*>(far_sh);
    double* ri = rr + NB * FARB_THREADS;
#pragma unroll
    for (int r = 0; r < NB; r++)
    {
        rr[r * FARB_THREADS + threadIdx.x] = accr[r];
        ri[r * FARB_THREADS + threadIdx.x] = acci[r];
    }
    __syncthreads();
    if (active && si == 0)
    {
        const long long o = a.tgt_perm[t];
        for (int r = 0; r < NB && pb + r < bp.nrhs; r++)
        {
            double sr = 0, sim = 0;
            for (int s = 0; s < S; s++)
            {
                sr += rr[r * FARB_THREADS + ti + s * cnt];
                sim += ri[r * FARB_THREADS + ti + s * cnt];
            }
            const double2 nr = bp.unear[(size_t)(pb + r) * bp.n_tgt + t];
            sr += nr.x;
            sim += nr.y;
            double* out = a.out + (size_t)(pb + r) * bp.out_plane;
            if (a.real_out)
                out[o] = sr;
            else
            {
                out[2 * o] = sr;
                out[2 * o + 1] = sim;
            }
        }
    }
}
