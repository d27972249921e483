// Far-field evaluation with coefficient blocks staged in shared memory, for
// the batched mixed pipeline (NP = BATCH_NB planes per CTA).  A single plane
// does not pay for the staging (the per-box work is a quarter, the hashing,
// copies and barriers are not): the single right-hand-side pipeline keeps its
// direct kernel.  Included by mult_kernels.cuh inside namespace ifgf, after
// the evaluation helpers.
#pragma once

// Far field of a plane group (blockIdx.y; NP planes): the cone lookup and the centred
// factor of a (target, far box) pair are computed once (with MK the factor
// once per plane); each plane's Chebyshev sum uses its own coefficient block.
// Adds the near sums and writes the caller's result planes (the first nrhs).
// Thread (ti, si) owns target ti and far boxes si, si + S, ... (S = threads /
// targets).  Coefficient blocks are staged in shared memory: for every S
// consecutive far boxes (one pair per thread) the CTA collects the distinct
// fine cones of its pairs in a small hash table, copies up to far_slots() of
// their 4-plane blocks with cp.async and evaluates from shared memory.  The
// lanes of a warp are targets of one leaf at one box, which fall into a few
// cones: from global memory every such load touches one sector per cone, from
// shared memory the few blocks are served together (slots start 16 bytes
// apart modulo 128, in different banks).  Pairs whose cone found no slot read
// global memory.  The evaluation order, and so the result, is that of the
// unstaged loop.
constexpr int FAR_HASH = 128;
template <int P_LO, int NP> __host__ __device__ constexpr int far_slot_stride()
{
    int s = NP * P_LO; // float2 per slot: NP planes, then pad to 16 B mod 128
    while ((s * 8) % 128 != 16 && (s * 8) % 128 != 80)
        s++;
    return s;
}
template <int P_LO, int NP> __host__ __device__ constexpr int far_slots()
{
    const int fit = 86016 / (far_slot_stride<P_LO, NP>() * 8); // about 84 KB: 2 CTAs per SM
    const int cap = 96 / NP; // within the hash table (FAR_HASH entries)
    return fit < cap ? fit : cap;
}
template <int N0, int N1, int N2, int NP> constexpr size_t far_batch_smem()
{
    constexpr size_t slots =
        (size_t)far_slots<N0 * N1 * N2, NP>() * far_slot_stride<N0 * N1 * N2, NP>() * 8;
    constexpr size_t red = 2 * NP * FAR_THREADS * sizeof(double); // final reduction
    return slots > red ? slots : red;
}

template <int KIND, int N0, int N1, int N2, bool MK, int NP>
__global__ void __launch_bounds__(FAR_THREADS, 2) far_batch_kernel(EvalArgs a, BatchPtrs bp)
{
    constexpr int NB = NP;
    constexpr int P_LO = N0 * N1 * N2;
    constexpr int SS = far_slot_stride<P_LO, NP>();
    constexpr int NSLOT = far_slots<P_LO, NP>();
    constexpr int CPP = P_LO / 2; // 16-byte chunks of one plane's block
    static_assert(P_LO % 2 == 0, "blocks must be whole 16-byte chunks");
    static_assert(NSLOT > 0, "one slot must fit");
    extern __shared__ __align__(16) float2 far_sh[]; // slots; the final reduction reuses it
    __shared__ int hkey[2][FAR_HASH], hslot[2][FAR_HASH], sgf[NSLOT], nslot[2];
    __shared__ KParams kps[MK ? NB : 1];
    const int pb = blockIdx.y * NB;
    if constexpr (MK)
        if (threadIdx.x < NB)
            kps[threadIdx.x] = bp.kp_plane[pb + threadIdx.x]; // read after the chunk barriers
    for (int q = threadIdx.x; q < 2 * FAR_HASH; q += blockDim.x)
        hkey[q / FAR_HASH][q % FAR_HASH] = -1;
    if (threadIdx.x < 2)
        nslot[threadIdx.x] = 0;
    __shared__ double fcx[FAR_THREADS], fcy[FAR_THREADS], fcz[FAR_THREADS], fH[FAR_THREADS];
    __shared__ long long ffm[FAR_THREADS];
    __shared__ int flev[FAR_THREADS];
    __shared__ LookupF lfs[MAX_LEVELS];
    for (int l = threadIdx.x; l < a.L; l += blockDim.x)
        make_lookupf(a.lv[l], lfs[l]); // read after the first chunk's barriers
    const int tl = blockIdx.x;
    const int tf = a.tl_first[tl], tlast = a.tl_last[tl];
    const long long fb0 = a.far_off[tl], fb1 = a.far_off[tl + 1];
    int tab = 0; // hash table of the current sub-chunk (CTA-uniform)
    for (int base = tf; base < tlast; base += FAR_THREADS)
    {
        const int cnt = min(FAR_THREADS, tlast - base);
        const int S = FAR_THREADS / cnt;
        const int ti = threadIdx.x % cnt, si = threadIdx.x / cnt;
        const bool active = si < S;
        const int t = base + ti;
        const double y0 = a.tx[t], y1 = a.ty[t], y2 = a.tz[t];
        double accr[NB], acci[NB];
#pragma unroll
        for (int r = 0; r < NB; r++)
            accr[r] = acci[r] = 0.0;
        for (long long e0 = fb0; e0 < fb1; e0 += FAR_THREADS)
        {
            const int fcnt = (int)min((long long)FAR_THREADS, fb1 - e0);
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
            // the cone of this thread's pair in sub-chunk box i (gf < 0: none)
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
            // sub-chunks of S boxes: at most one pair per thread; every
            // thread runs every sub-chunk (barriers inside).  The next
            // sub-chunk's lookup (a dependent global load) is issued before
            // this one's copies are waited for.
            for (int c0 = 0; c0 < fcnt; c0 += S)
            {
                const int gf = gf_next;
                const float loc[3] = {loc_next[0], loc_next[1], loc_next[2]};
                const double d2 = d2_next;
                int h = -1;
                if (gf >= 0)
                {
                    // insert the cone, bounded linear probing; the first
                    // inserter takes a slot while slots last
                    int hh = (int)(((unsigned)gf * 2654435761u) >> 25) & (FAR_HASH - 1);
                    for (int q = 0; q < FAR_HASH; q++, hh = (hh + 1) & (FAR_HASH - 1))
                    {
                        const int prev = atomicCAS(&hkey[tab][hh], -1, gf);
                        if (prev == -1)
                        {
                            const int k = atomicAdd(&nslot[tab], 1);
                            if (k < NSLOT)
                                sgf[k] = gf;
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
                }
                __syncthreads(); // table and slot list complete
                const int ns = min(nslot[tab], NSLOT);
                // the other table was last read before this barrier: clear it
                for (int q = threadIdx.x; q < FAR_HASH; q += blockDim.x)
                    hkey[tab ^ 1][q] = -1;
                if (threadIdx.x == 0)
                    nslot[tab ^ 1] = 0;
                // one warp per slot, lanes over the slot's 16-byte chunks
                for (int k = threadIdx.x >> 5; k < ns; k += FAR_THREADS / 32)
                {
                    const float2* src0 = bp.fcoef + (size_t)pb * bp.fc_plane + (size_t)sgf[k] * P_LO;
                    float2* dst0 = far_sh + (size_t)k * SS;
#pragma unroll
                    for (int r = 0; r < NB; r++)
                        for (int ch = threadIdx.x & 31; ch < CPP; ch += 32)
                            cp_async16(dst0 + r * P_LO + 2 * ch,
                                       src0 + (size_t)r * bp.fc_plane + 2 * ch);
                }
                lookup(c0 + S + si, gf_next, loc_next, d2_next);
                cp_async_wait_all();
                __syncthreads(); // blocks staged
                if (gf >= 0)
                {
                    const int k = h >= 0 ? hslot[tab][h] : -1;
                    cplx<float> cf;
                    if constexpr (!MK)
                        cf = cf_mixed<KIND>(d2, a.kp);
#pragma unroll
                    for (int r = 0; r < NB; r++)
                    {
                        if constexpr (MK)
                            cf = cf_mixed<KIND>(d2, kps[r]);
                        const cplx<float> v =
                            k >= 0 ? ChebF<N0, N1, N2, true>::eval(far_sh + (size_t)k * SS +
                                                                       r * P_LO,
                                                                   loc, a.lo)
                                   : ChebF<N0, N1, N2>::eval(bp.fcoef +
                                                                 (size_t)(pb + r) * bp.fc_plane +
                                                                 (size_t)gf * P_LO,
                                                             loc, a.lo);
                        accr[r] += (double)(v.re * cf.re - v.im * cf.im);
                        acci[r] += (double)(v.re * cf.im + v.im * cf.re);
                    }
                }
                tab ^= 1;
            }
        }
        __syncthreads(); // the slots are no longer read: reduce through them
        double* rr = reinterpret_cast<double*>(far_sh);
        double* ri = rr + NB * FAR_THREADS;
#pragma unroll
        for (int r = 0; r < NB; r++)
        {
            rr[r * FAR_THREADS + threadIdx.x] = accr[r];
            ri[r * FAR_THREADS + threadIdx.x] = acci[r];
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
                    sr += rr[r * FAR_THREADS + ti + s * cnt];
                    sim += ri[r * FAR_THREADS + ti + s * cnt];
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

