// IFGF operator: init (host planner + GPU active-cone tables) and the host side
// of mult.  The matvec kernels themselves are in mult_kernels.cuh.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <sstream>

#include "devbuf.hpp"
#include "device_math.cuh"
#include "gpu_target_lists.hpp"
#include "tcgen05.cuh"
#include "mult.hpp"
#include "operator.hpp"

namespace ifgf
{

// Calls CALL with the compile-time kernel kind KK matching KINDVAR.
#define IFGF_DISPATCH(KINDVAR, CALL)                                                          \
    switch (KINDVAR)                                                                           \
    {                                                                                          \
    case K_LAPLACE: { constexpr int KK = K_LAPLACE; CALL; } break;                            \
    case K_HELMHOLTZ: { constexpr int KK = K_HELMHOLTZ; CALL; } break;                        \
    case K_MODHELMHOLTZ: { constexpr int KK = K_MODHELMHOLTZ; CALL; } break;                  \
    case K_GRADHELMHOLTZ: { constexpr int KK = K_GRADHELMHOLTZ; CALL; } break;                \
    case K_DOUBLELAYER: { constexpr int KK = K_DOUBLELAYER; CALL; } break;                    \
    case K_COMBINEDFIELD: { constexpr int KK = K_COMBINEDFIELD; CALL; } break;                \
    case K_HELMHOLTZ_DK: { constexpr int KK = K_HELMHOLTZ_DK; CALL; } break;                  \
    case K_COMBINEDFIELD_DK: { constexpr int KK = K_COMBINEDFIELD_DK; CALL; } break;          \
    }

struct DeviceState
{
    DevBuf<LevelGeom> lv;
    DevBuf<double> box_c, box_H;
    DevBuf<int> box_first, box_last, box_child, box_level;
    DevBuf<unsigned char> box_leaf;
    DevBuf<double> sx, sy, sz, nx, ny, nz, tx, ty, tz;
    DevBuf<long long> src_perm, tgt_perm;
    std::vector<DevBuf<int>> cc_box, cc_el, fc_box, fc_el; // per level
    std::vector<DevBuf<int>> leaf_idx, up_idx, up_slot;    // per level coarse-cone partition
    std::vector<DevBuf<UpGeo64>> geo64;                    // per level upward geometry
    std::vector<DevBuf<UpGeo32>> geo32;
    std::vector<DevBuf<int2>> fe_list; // per-row (child element, first group) of each run
    std::vector<DevBuf<int>> c2f_idx;  // per level: coarse cones of a sharded operator
    // what the upward geometry of a level is built from (kept for variants)
    std::vector<DevBuf<int>> slot_el;      // element of each slot
    std::vector<DevBuf<double>> child_off; // 8 child-centre offsets
    std::vector<double> up_pH, up_cH;      // parent / child side lengths
    // variant kernel (k-derivative) geometry tables and list views
    int vkind = -1;
    std::vector<DevBuf<UpGeo64>> vgeo64;
    std::vector<DevBuf<UpGeo32>> vgeo32;
    std::vector<LevelLists> vlists;
    std::vector<LevelLists> lists;                         // per level views of the above
    DevBuf<int> fmap;
    DevBuf<double> hi_nodes, A;
    std::vector<double> A_host; // host copy of A
    DevBuf<int> tl_first, tl_last, tl_far_src, tl_near_src;
    DevBuf<long long> tl_far_off, tl_near_off;
    // far-field plan of the batched mixed matvec (built on first use)
    DevBuf<FarChunk> fp_chunk;
    DevBuf<FarGroup> fp_group;
    DevBuf<FarPlanRec> fp_rec;
    DevBuf<int> fp_slot;
    int fp_nchunk = 0;
    int fp_nslot = 0;
    double fp_ovf_few = 0; // share of the records beyond the smaller slot count tried
    bool fp_ready = false;
    double fp_ms = 0;
    DevBuf<double2> w, cvals, fcoef, unear;
    // planes of the batched mixed matvec, allocated on first use for
    // b_planes planes of the plane sizes recorded beside them
    DevBuf<float2> bw, bcv, bfc;
    DevBuf<double2> bun;
    int b_planes = 0;
    size_t b_cv = 0, b_fc = 0;
    int64_t b_ns = 0, b_nt = 0;
    // multi-wavenumber batches: per-plane wavenumbers and the per-level
    // distance tables (built on first use after an init)
    DevBuf<KParams> kp_plane;
    std::vector<KParams> kp_host; // what kp_plane holds
    std::vector<DevBuf<UpGeo32>> dgeo32;
    std::vector<const UpGeo32*> dgeo32_ptr;
    bool dgeo_ready = false;
    DevBuf<unsigned long long> err;
    // tensor-core upward transfer: per level the runs of equal slots in
    // up_idx order (first position, cones); row tiles and their fill per
    // plane count of a launch; the per-level views handed to a batch; the
    // status word of the kernels' bounded waits
    std::vector<std::vector<int2>> tc_runs;
    std::vector<std::map<int, DevBuf<int4>>> tc_tiles;
    // basis images of the tensor-core upward transfer, per level (built on
    // first use of the mixed pipeline; empty where not worth their memory)
    std::vector<DevBuf<unsigned char>> tc_img;
    std::vector<DevBuf<long long>> tc_img_off;
    bool tc_img_ready = false;
    std::vector<std::map<int, float>> tc_fill;
    std::vector<const int4*> tcb_ptr;
    std::vector<int> tcb_n;
    std::vector<float> tcb_fill;
    DevBuf<unsigned> tc_status;
    // upward-kernel autotuner: per plane count of a launch, the per-level
    // choice (1 tensor cores, 0 FFMA, -1 not both) and the timed milliseconds
    std::map<int, std::vector<signed char>> up_choice;
    std::map<int, std::vector<double>> up_ms_ffma, up_ms_tc;
    DevBuf<double> io_w, io_u; // staging for host-buffer mult
    std::vector<cudaEvent_t> prof_ev;
    cudaStream_t side = nullptr; // near-field stream
    // pipelined host-buffer batches: compute, upload and download streams,
    // and two events per group of right-hand sides
    cudaStream_t io_cs = nullptr, io_up = nullptr, io_down = nullptr;
    std::vector<cudaEvent_t> io_ev;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int n_tleaf = 0;
    size_t c2f_smem = 0;
    ~DeviceState()
    {
        for (auto& e : prof_ev)
            cudaEventDestroy(e);
        if (ev_fork)
            cudaEventDestroy(ev_fork);
        if (ev_join)
            cudaEventDestroy(ev_join);
        if (side)
            cudaStreamDestroy(side);
        for (auto& e : io_ev)
            cudaEventDestroy(e);
        for (cudaStream_t st : {io_cs, io_up, io_down})
            if (st)
                cudaStreamDestroy(st);
    }
};

// Operators and buffers of the adjoint (see Operator::mult_adjoint_device).
struct AdjointState
{
    // 0: conj(A conj w) on this operator; 1: sign conj(A' conj w) on the
    // swapped operator; 2: double layer; 3: combined field
    int mode = -1;
    double sign = 1;
    std::vector<std::unique_ptr<Operator>> ops;
    DevBuf<double2> wc;    // conj(w)
    DevBuf<double2> z[4];  // results of the swapped operators
    DevBuf<double> nx, ny, nz; // source normals in the caller's order
    DevBuf<double> io_w, io_u; // host-buffer staging
};

// ---------------------------------------------------------------------------
// Setup kernels: active-cone marking (octree.hpp:571-690) and compaction
// ---------------------------------------------------------------------------
// One CTA per far pair (source box, target range): mark the fine and coarse
// cones that contain the far targets (octree.hpp:574-590).
__global__ void mark_far_kernel(LevelGeom G, TreeArgs T, const int* __restrict__ fp_src,
                                const int* __restrict__ fp_tgt, const int* __restrict__ tbox_first,
                                const int* __restrict__ tbox_last, const double* __restrict__ tx,
                                const double* __restrict__ ty, const double* __restrict__ tz,
                                int* fmark, int* cmark)
{
    const int pr = blockIdx.x;
    const int sb = fp_src[pr];
    const int tb = fp_tgt[pr];
    const int lb = sb - G.box_off;
    const double xc0 = T.box_c[3 * sb], xc1 = T.box_c[3 * sb + 1], xc2 = T.box_c[3 * sb + 2];
    const double H = T.box_H[sb];
    const long long nf = (long long)G.nf[0] * G.nf[1] * G.nf[2];
    const long long nc = (long long)G.nc[0] * G.nc[1] * G.nc[2];
    const int t1 = tbox_last[tb];
    for (int t = tbox_first[tb] + threadIdx.x; t < t1; t += blockDim.x)
    {
        double s[3];
        cart_to_interp(tx[t] - xc0, ty[t] - xc1, tz[t] - xc2, H, s);
        const int fe = element_for_point(s, G.dmin, G.dmax, G.hfi, G.nf);
        const int ce = element_for_point(s, G.dmin, G.dmax, G.hci, G.nc);
        if (fe >= 0)
            fmark[G.fmap_off + lb * nf + fe] = 1;
        if (ce >= 0)
            cmark[lb * nc + ce] = 1;
    }
}

// Far-field plan (FarChunk / FarGroup / FarPlanRec, mult.hpp): one CTA per
// chunk of up to 256 targets of a target leaf, thread (ti, si) = target ti,
// far box si of each group of S = 256 / targets consecutive boxes of the
// leaf's far list (evaluateFromInterp's pairs, ifgfoperator.hpp:1736-1891).
// Per group: the fine cone and local coordinates of every pair (the lookup
// of the far kernels), the distinct cones in a hash table of twice the pairs
// (never full, so every cone is in it), slots for the nslot cones with the
// most pairs (ties: smaller id first), and the records in slot order, each
// slot's run padded
// to FAR_PLAN_PAD positions; pairs of the other cones go last, with their cone ids
// after the group's slot list.  Every count depends only on the set of cones
// of the group, not on the order of the atomics, so the two passes agree:
// FILL = false counts the groups, records and slot-list entries of every
// chunk (and the pairs beyond the slots, which read global memory); FILL =
// true writes them at the offsets the counts gave and reports its own
// totals, which the host compares.
struct FarBuildArgs
{
    const LevelGeom* lv;
    int L;
    const double* box_c;
    const double* box_H;
    const int* box_level;
    const double *tx, *ty, *tz;
    const int* fmap;
    const long long* far_off;
    const int* far_src;
    const int* c_leaf;
    const int* c_t0;
    const int* c_cnt;
    unsigned long long* err;
    int nslot; // slots per group, <= FAR_PLAN_SLOTS
    long long *n_group, *n_rec, *n_slot, *n_ovf;             // counting pass
    const long long *g_off, *rec_off, *slot_off;     // filling pass
    FarGroup* group;
    FarPlanRec* rec;
    int* slot;
};

template <bool FILL>
__global__ void __launch_bounds__(256) far_plan_build_kernel(FarBuildArgs b)
{
    constexpr int T = 256, H = 2 * T, NBOX = 128;
    const int NS = b.nslot;
    __shared__ int hkey[H], hcnt[H], hrank[H];
    __shared__ int klist[T], kent[T]; // distinct cones, their table entries
    __shared__ int sgf[FAR_PLAN_SLOTS], scnt[FAR_PLAN_SLOTS];
    __shared__ int ndist, novf;
    __shared__ double fcx[NBOX], fcy[NBOX], fcz[NBOX], fH[NBOX];
    __shared__ long long ffm[NBOX];
    __shared__ int flev[NBOX];
    __shared__ LookupF lfs[MAX_LEVELS];
    const int c = blockIdx.x;
    const int tl = b.c_leaf[c], t0 = b.c_t0[c], cnt = b.c_cnt[c];
    const int S = T / cnt, ti = threadIdx.x % cnt, si = threadIdx.x / cnt;
    const bool active = si < S;
    const int lane = threadIdx.x & 31;
    for (int l = threadIdx.x; l < b.L; l += T)
        make_lookupf(b.lv[l], lfs[l]);
    for (int e = threadIdx.x; e < H; e += T)
    {
        hkey[e] = -1;
        hcnt[e] = 0;
    }
    if (threadIdx.x == 0)
        ndist = novf = 0;
    const double y0 = b.tx[t0 + ti], y1 = b.ty[t0 + ti], y2 = b.tz[t0 + ti];
    const long long fb0 = b.far_off[tl], fb1 = b.far_off[tl + 1];
    long long gi = FILL ? b.g_off[c] : 0, ri = FILL ? b.rec_off[c] : 0,
              sl = FILL ? b.slot_off[c] : 0;
    long long ovf = 0; // pairs beyond the slots
    for (long long e0 = fb0; e0 < fb1; e0 += NBOX)
    {
        const int fcnt = (int)min((long long)NBOX, fb1 - e0);
        __syncthreads();
        if (threadIdx.x < fcnt)
        {
            const int sb = b.far_src[e0 + threadIdx.x];
            const int lev = b.box_level[sb];
            const LevelGeom& G = b.lv[lev];
            const long long nft = (long long)G.nf[0] * G.nf[1] * G.nf[2];
            fcx[threadIdx.x] = b.box_c[3 * sb];
            fcy[threadIdx.x] = b.box_c[3 * sb + 1];
            fcz[threadIdx.x] = b.box_c[3 * sb + 2];
            fH[threadIdx.x] = b.box_H[sb];
            ffm[threadIdx.x] = G.fmap_off + (long long)(sb - G.box_off) * nft;
            flev[threadIdx.x] = lev;
        }
        __syncthreads();
        for (int c0 = 0; c0 < fcnt; c0 += S)
        {
            const int i = c0 + si;
            int gf = -1;
            float loc[3] = {0.f, 0.f, 0.f};
            if (active && i < fcnt)
            {
                const int lev = flev[i];
                const double p[3] = {y0 - fcx[i], y1 - fcy[i], y2 - fcz[i]};
                gf = fine_lookup_fast(lfs[lev], b.lv[lev], b.fmap + ffm[i], p, fH[i], loc, b.err);
            }
            int h = -1, rank = 0;
            if (gf >= 0)
            {
                int hh = (int)(((unsigned)gf * 2654435761u) >> 23) & (H - 1);
                for (int q = 0; q < H; q++, hh = (hh + 1) & (H - 1))
                {
                    const int prev = atomicCAS(&hkey[hh], -1, gf);
                    if (prev == -1)
                    {
                        const int id = atomicAdd(&ndist, 1);
                        klist[id] = gf;
                        kent[id] = hh;
                    }
                    if (prev == -1 || prev == gf)
                    {
                        h = hh;
                        break;
                    }
                }
                rank = atomicAdd(&hcnt[h], 1); // the table has room for every pair
            }
            __syncthreads(); // table, cone list and counts complete
            const int nd = ndist;
            if (threadIdx.x < nd)
            {
                // rank by pairs (most first), then cone id: the slots hold the
                // most-used cones, so the fewest pairs read global memory
                const int key = klist[threadIdx.x], kc = hcnt[kent[threadIdx.x]];
                int r = 0;
                for (int u = 0; u < nd; u++)
                {
                    const int cu = hcnt[kent[u]];
                    r += cu > kc || (cu == kc && klist[u] < key) ? 1 : 0;
                }
                hrank[kent[threadIdx.x]] = r;
                if (r < NS)
                {
                    sgf[r] = key;
                    scnt[r] = kc;
                }
            }
            __syncthreads(); // slot order complete
            const int ns = min(nd, NS);
            const int ck = lane < ns ? scnt[lane] : 0;
            const int pk = (ck + FAR_PLAN_PAD - 1) & ~(FAR_PLAN_PAD - 1);
            int incl = pk;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1)
            {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o)
                    incl += v;
            }
            const int slotted = __shfl_sync(0xffffffffu, incl, 31);
            const int k = h >= 0 ? hrank[h] : -1;
            const bool in_slot = k >= 0 && k < NS;
            const int src = in_slot ? k : 0;
            const int kbase = __shfl_sync(0xffffffffu, incl - pk, src);
            const int kcnt = __shfl_sync(0xffffffffu, ck, src);
            const int kend = __shfl_sync(0xffffffffu, incl, src);
            int pos = -1;
            if (gf >= 0)
                pos = in_slot ? kbase + rank : slotted + atomicAdd(&novf, 1);
            __syncthreads(); // overflow count complete
            const int nov = novf;
            if (FILL)
            {
                if (gf >= 0)
                {
                    b.rec[ri + pos] =
                        FarPlanRec{__float_as_int(loc[0]), __float_as_int(loc[1]),
                                   __float_as_int(loc[2]),
                                   (int)threadIdx.x | ((in_slot ? k : FAR_PLAN_OVF) << 9)};
                    if (in_slot && rank == kcnt - 1)
                        for (int q = kbase + kcnt; q < kend; q++)
                            b.rec[ri + q] = FarPlanRec{0, 0, 0, FAR_PLAN_PAD_OWNER | (k << 9)};
                    if (!in_slot)
                        b.slot[sl + ns + (pos - slotted)] = gf;
                }
                if (threadIdx.x < ns)
                    b.slot[sl + threadIdx.x] = sgf[threadIdx.x];
                if (threadIdx.x == 0)
                {
                    FarGroup G;
                    G.rec = ri;
                    G.box0 = e0 + c0;
                    G.slot = (int)sl;
                    G.npos = (unsigned short)(slotted + nov);
                    G.nslotted = (unsigned short)slotted;
                    G.nbox = (unsigned short)min(S, fcnt - c0);
                    G.nslot = (unsigned char)ns;
                    G.pad_ = 0;
                    b.group[gi] = G;
                }
            }
            gi++;
            ri += slotted + nov;
            sl += ns + nov;
            ovf += nov;
            __syncthreads(); // the table is read no more: clear it
            for (int e = threadIdx.x; e < H; e += T)
            {
                hkey[e] = -1;
                hcnt[e] = 0;
            }
            if (threadIdx.x == 0)
                ndist = novf = 0;
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) // FILL: the end offsets, which the host checks
    {
        b.n_group[c] = gi;
        b.n_rec[c] = ri;
        b.n_slot[c] = sl;
        b.n_ovf[c] = ovf;
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
            const int fe = element_for_point(s2, G.dmin, G.dmax, G.hfi, G.nf);
            const int ce = element_for_point(s2, G.dmin, G.dmax, G.hci, G.nc);
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
    if (dx != dx_)
        adj_.reset(); // the adjoint of the gradient kernel follows dx
    dx_ = dx;
}

void Operator::set_wavenumber(double k_re, double k_im)
{
    if (!std::isfinite(k_re) || !std::isfinite(k_im))
        throw Error(ERR_INVALID, "wavenumber must be finite");
    if (!initialized_)
    {
        kr_ = k_re;
        ki_ = k_im;
        return;
    }
    const double okr = kr_, oki = ki_;
    bool same = grids_match(k_re, k_im);
    kr_ = k_re;
    ki_ = k_im;
    if (same && tol_ > 0)
    {
        // estimated orders follow the wavenumber: new orders need a new init
        int est[3];
        estimate_orders(est);
        for (int d = 0; d < 3; d++)
            same = same && est[d] == base_order_[d];
    }
    adj_.reset();
    if (!same)
    {
        // new cone grids: a full init from the stored points
        const std::vector<double> s = src_pts_, t = tgt_pts_, nrm = normals_;
        const auto cut = cutoff_;
        try
        {
            init(s.data(), (int64_t)s.size() / 3, t.data(), (int64_t)t.size() / 3,
                 nrm.empty() ? nullptr : nrm.data(), cut);
        }
        catch (...)
        {
            kr_ = okr;
            ki_ = oki;
            throw;
        }
        return;
    }
    DeviceState& D = *dev_;
    const int L = (int)lv_.size();
    const int P_hi = hi_[0] * hi_[1] * hi_[2];
    const KParams kp = make_kparams(kr_, ki_, dx_);
    for (int l = 0; l + 1 < L; l++)
    {
        const LevelLists& LL = D.lists[l];
        const int ns = (int)D.slot_el[l].n;
        if (ns == 0 || LL.up_pad <= 0)
            continue;
        const size_t n_ent = (size_t)ns * 8 * (size_t)LL.up_pad;
        IFGF_CUDA(cudaMemset(D.geo64[l].p, 0xff, n_ent * sizeof(UpGeo64)));
        IFGF_CUDA(cudaMemset(D.geo32[l].p, 0xff, n_ent * sizeof(UpGeo32)));
        IFGF_DISPATCH(kind_, launch_build_upgeo<KK>(lv_[l], lv_[l + 1], D.up_pH[l], D.up_cH[l],
                                                     D.child_off[l].p, D.slot_el[l].p, ns,
                                                     D.hi_nodes.p, P_hi, kp, LL.up_pad,
                                                     D.geo64[l].p, D.geo32[l].p, LL.fe_pad,
                                                     D.fe_list[l].p));
    }
    IFGF_CUDA(cudaDeviceSynchronize());
    D.vkind = -1; // variant (k-derivative) tables are rebuilt on next use
    // the basis images hold the old centre-shift factors: new entry data (the
    // basis rows do not depend on the wavenumber)
    for (int l = 0; l < (int)D.tc_img.size(); l++)
        if (D.tc_img[l].n > 0)
        {
            const LevelLists& LL = D.lists[l];
            upward_tc_image_fill(lo_, LL.fe_list, LL.fe_pad, LL.geo32, LL.up_pad,
                                 (int)D.slot_el[l].n, D.tc_img_off[l].p, D.tc_img[l].p, true);
        }
}

// Whether wavenumber k_re + i k_im gives every level the cone grids and
// interpolation domain the operator was initialised with.
bool Operator::grids_match(double k_re, double k_im)
{
    const double okr = kr_, oki = ki_;
    kr_ = k_re;
    ki_ = k_im;
    bool same = true;
    for (const LevelGeom& G : lv_)
    {
        int64_t nf[3], nc[3];
        elements_for_box(G.H, 0, nf);
        elements_for_box(G.H, 1, nc);
        double smin = cutoff_limit(G.H);
        if (smin >= std::sqrt(3.0) / 3)
            smin = std::sqrt(3.0) / 3 - 0.05;
        for (int d = 0; d < 3; d++)
            same = same && nf[d] == G.nf[d] && nc[d] == G.nc[d];
        same = same && smin == G.dmin[0];
    }
    kr_ = okr;
    ki_ = oki;
    return same;
}

void Operator::set_shard(int rank, int nranks)
{
    if (nranks < 1 || rank < 0 || rank >= nranks)
        throw Error(ERR_INVALID, "shard rank must be in [0, nranks)");
    shard_rank_ = rank;
    shard_n_ = nranks;
    initialized_ = planned_ = false; // takes effect at the next init
}

std::vector<int64_t> Operator::shard_boxes() const
{
    std::vector<int64_t> out;
    if (!planned_ && !initialized_)
        throw Error(ERR_STATE, "shard boxes are known after init");
    const int S = plan_.shard_level;
    const int64_t off = plan_.src.level_off[S];
    for (size_t b = 0; b < plan_.src.levels[S].size(); b++)
        if (plan_.box_rank[off + (int64_t)b] == shard_rank_)
            out.push_back((int64_t)b);
    return out;
}

void Operator::set_precision(int mode)
{
    if (mode != PREC_FP64 && mode != PREC_MIXED)
        throw Error(ERR_INVALID, "precision must be FP64 (0) or MIXED (1)");
    // the fine-coefficient buffer changes element type: cones that are never
    // written (no active coarse parent) must read zero in the new layout
    if (mode != precision_ && initialized_)
        dev_->fcoef.zero();
    precision_ = mode;
    if (adj_)
        for (auto& op : adj_->ops)
            op->set_precision(mode);
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

// Low (step 0) and high (step 1) orders from base_order_, within what the
// kernels support.
void Operator::set_orders()
{
    order_for_box(0, lo_);
    order_for_box(1, hi_);
    for (int i = 0; i < 3; i++)
        if (lo_[i] < 1 || hi_[i] < 1)
            throw Error(ERR_INVALID, "interpolation order too low for this kernel (the low-order "
                                     "grid would have order < 1; use order >= 7)");
    if (lo_[0] * lo_[1] * lo_[2] > 4096 || hi_[0] * hi_[1] * hi_[2] > 2048 || lo_[0] > 16 ||
        lo_[1] > 16 || lo_[2] > 16)
        throw Error(ERR_INVALID, "interpolation order too high");
}

// estimateRefinement / estimateRefinementOnBox with RefineP
// (ifgfoperator.hpp:108-244).  Ten boxes spaced Nboxes/10 apart on the
// deepest source level; in each, the order of a dimension grows by one while
// the Chebyshev layer n - 3 of the order + 4 expansion of the box's factored
// kernel (unit weights) on coarse cone 0 holds more than tol of the
// coefficient norm, at most 10 times; the result is the component-wise
// maximum over the boxes.  Kernel values come from order_probe_kernel (all
// live samples in one launch per step); the transform and the norms are a
// few thousand host operations per step.
// The reference draws the cone as (n_elements * Random()) / SIZE_MAX in
// size_t arithmetic, which is 0 for every draw (the product stays below
// SIZE_MAX or wraps below it); its TBB reduction keeps only the last box of
// each subrange it is handed, which equals the maximum over all ten boxes
// when every subrange holds one box.
void Operator::estimate_orders(int* out) const
{
    constexpr int SAMPLES = 10, MAX_R = 10, LAYERS = 3;
    const Tree& S = plan_.src;
    const TreeLevel& TL = S.levels[S.num_levels() - 1];
    const int64_t stride = (int64_t)TL.size() / SAMPLES;
    const bool need_n = kind_ == K_DOUBLELAYER || kind_ == K_COMBINEDFIELD;
    if (need_n && normals_.size() != 3 * (size_t)S.n)
        throw Error(ERR_INVALID, "this kernel needs source normals");
    std::vector<double> sc[6];
    std::vector<int> src_off(SAMPLES + 1, 0);
    std::vector<double> centre(3 * SAMPLES);
    double H[SAMPLES];
    for (int i = 0; i < SAMPLES; i++)
    {
        const int64_t b = i * stride;
        for (int d = 0; d < 3; d++)
            centre[3 * i + d] = TL.center[3 * b + d];
        H[i] = TL.sides[b];
        for (int64_t j = TL.first[b]; j < TL.last[b]; j++)
            for (int d = 0; d < 3; d++)
            {
                sc[d].push_back(S.pts[3 * j + d]);
                sc[3 + d].push_back(need_n ? normals_[3 * S.perm[j] + d] : 0.0);
            }
        src_off[i + 1] = (int)sc[0].size();
    }
    DevBuf<double> d_sc[6], d_centre, d_nodes;
    DevBuf<int> d_src_off, d_node_off;
    DevBuf<double2> d_vals;
    for (int d = 0; d < 6; d++)
        d_sc[d].upload(sc[d].data(), sc[d].size());
    d_centre.upload(centre.data(), centre.size());
    d_src_off.upload(src_off.data(), src_off.size());

    int base[SAMPLES][3] = {}, newp[SAMPLES][3], order[SAMPLES][3];
    double err[SAMPLES][3];
    bool live[SAMPLES];
    for (int i = 0; i < SAMPLES; i++)
    {
        live[i] = true;
        for (int d = 0; d < 3; d++)
            err[i][d] = std::numeric_limits<double>::max();
    }
    for (;;)
    {
        std::vector<double> nodes;
        std::vector<int> node_off(SAMPLES + 1, 0);
        int max_nodes = 0;
        for (int i = 0; i < SAMPLES; i++)
        {
            if (live[i])
            {
                for (int d = 0; d < 3; d++)
                {
                    newp[i][d] = order0_ + base[i][d];
                    order[i][d] = newp[i][d] + LAYERS + 1; // orderForBox(step 1) is the identity
                }
                int64_t ne[3];
                elements_for_box(H[i], 1, ne);
                // interpolation box [cutoff_limit(H), sqrt(3)/3] x [0, pi] x [-pi, pi]; a
                // reversed one gives unit element sizes (ConeDomain, cone_domain.hpp:72-83)
                const double mn[3] = {cutoff_limit(H[i]), 0.0, -M_PI};
                const double mx[3] = {std::sqrt(3.0) / 3, M_PI, M_PI};
                const bool null_box = mn[0] > mx[0];
                double a[3], b[3];
                for (int d = 0; d < 3; d++)
                {
                    const double h = null_box ? 1.0 : (mx[d] - mn[d]) / (double)ne[d];
                    a[d] = 0.5 * h;
                    b[d] = mn[d] + 0.5 * h; // cone 0
                }
                std::vector<double> x[3];
                for (int d = 0; d < 3; d++)
                    for (int q = 0; q < order[i][d]; q++)
                        x[d].push_back(std::cos((2. * q + 1.0) / (2. * order[i][d]) * M_PI));
                for (int i2 = 0; i2 < order[i][2]; i2++)
                    for (int i1 = 0; i1 < order[i][1]; i1++)
                        for (int i0 = 0; i0 < order[i][0]; i0++)
                        {
                            const double s0 = x[0][i0] * a[0] + b[0], s1 = x[1][i1] * a[1] + b[1],
                                         s2 = x[2][i2] * a[2] + b[2];
                            const double r = H[i] / s0; // util.hpp:96-116
                            nodes.push_back(centre[3 * i] + r * std::cos(s2) * std::sin(s1));
                            nodes.push_back(centre[3 * i + 1] + r * std::sin(s2) * std::sin(s1));
                            nodes.push_back(centre[3 * i + 2] + r * std::cos(s1));
                        }
            }
            node_off[i + 1] = (int)(nodes.size() / 3);
            max_nodes = std::max(max_nodes, node_off[i + 1] - node_off[i]);
        }
        if (max_nodes == 0)
            break;
        d_nodes.upload(nodes.data(), nodes.size());
        d_node_off.upload(node_off.data(), node_off.size());
        d_vals.alloc(nodes.size() / 3);
        ProbeArgs pa;
        pa.S = SrcArgs{d_sc[0].p, d_sc[1].p, d_sc[2].p, d_sc[3].p, d_sc[4].p, d_sc[5].p};
        pa.src_off = d_src_off.p;
        pa.nodes = d_nodes.p;
        pa.node_off = d_node_off.p;
        pa.centre = d_centre.p;
        pa.kp = make_kparams(kr_, ki_, dx_);
        pa.out = d_vals.p;
        IFGF_DISPATCH(kind_, launch_order_probe<KK>(pa, SAMPLES, max_nodes, 0));
        std::vector<double2> vals(nodes.size() / 3);
        IFGF_CUDA(cudaMemcpy(vals.data(), d_vals.p, vals.size() * sizeof(double2),
                             cudaMemcpyDeviceToHost));
        for (int i = 0; i < SAMPLES; i++)
        {
            if (!live[i])
                continue;
            const int* n = order[i];
            const size_t np = (size_t)n[0] * n[1] * n[2];
            // chebtransform (chebinterp.hpp:176-250): one dimension at a time,
            // c_k = (k ? 2 : 1) / n sum_j v_j cos(k pi (2 j + 1) / (2 n))
            std::vector<std::complex<double>> c(np), t(np);
            for (size_t q = 0; q < np; q++)
                c[q] = {vals[node_off[i] + q].x, vals[node_off[i] + q].y};
            size_t inner = 1;
            for (int d = 0; d < 3; d++)
            {
                const int nd = n[d];
                const size_t outer = np / (inner * nd);
                for (size_t o = 0; o < outer; o++)
                    for (size_t in = 0; in < inner; in++)
                        for (int k = 0; k < nd; k++)
                        {
                            std::complex<double> acc = 0;
                            for (int j = 0; j < nd; j++)
                                acc += c[(o * nd + j) * inner + in] *
                                       std::cos(k * M_PI * (2. * j + 1) / (2. * nd));
                            t[(o * nd + k) * inner + in] = acc * ((k ? 2.0 : 1.0) / nd);
                        }
                std::swap(c, t);
                inner *= nd;
            }
            // Util::compute_slice_norm (util.hpp:214-234)
            double v1 = 0, v2[3] = {0, 0, 0};
            for (size_t q = 0; q < np; q++)
            {
                const double m2 = std::norm(c[q]);
                v1 += m2;
                const size_t id[3] = {q % n[0], (q / n[0]) % n[1], q / ((size_t)n[0] * n[1])};
                for (int d = 0; d < 3; d++)
                    if ((int)id[d] == n[d] - LAYERS)
                        v2[d] += m2;
            }
            for (int d = 0; d < 3; d++)
            {
                err[i][d] = std::sqrt(v2[d]) / std::max(1., std::sqrt(v1));
                if (err[i][d] > tol_)
                    base[i][d] += 1;
            }
            live[i] = std::max(err[i][0], std::max(err[i][1], err[i][2])) > tol_ &&
                      std::max(base[i][0], std::max(base[i][1], base[i][2])) < MAX_R;
        }
    }
    for (int d = 0; d < 3; d++)
    {
        out[d] = 0;
        for (int i = 0; i < SAMPLES; i++)
            out[d] = std::max(out[d], newp[i][d]);
    }
}

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
    if (tol_ > 0 && plan_only)
        throw Error(ERR_INVALID, "order estimation (tol > 0) samples the kernel on the GPU; a "
                                 "plan-only init needs tol <= 0");
    // fixed-order path: radial order reset of ifgfoperator.hpp:90, taken from
    // the constructor's order so that a repeated init does not compound it;
    // with tol > 0 the orders are estimated once the source octree exists
    base_order_[0] = std::max(order0_ - 3, 2);
    base_order_[1] = base_order_[2] = order0_;
    if (tol_ <= 0)
        set_orders();

    adj_.reset();
    src_pts_.assign(srcs, srcs + 3 * ns);
    tgt_pts_.assign(tgts, tgts + 3 * nt);
    if (normals)
        normals_.assign(normals, normals + 3 * ns);
    else
        normals_.clear();
    cutoff_ = cutoff;
    same_points_ = ns == nt && std::equal(srcs, srcs + 3 * ns, tgts);
    plan_ = Plan();
    // the octrees on the GPU; a plan-only init (no GPU needed) on the host,
    // with the same result
    const auto tt0 = std::chrono::steady_clock::now();
    if (plan_only)
    {
        plan_.src.build(srcs, ns, leaf_);
        plan_.tgt.build(tgts, nt, leaf_);
    }
    else
    {
        plan_.src.build_gpu(srcs, ns, leaf_);
        if (same_points_ && ns == nt)
            plan_.tgt = plan_.src;
        else
            plan_.tgt.build_gpu(tgts, nt, leaf_);
    }
    const auto tt1 = std::chrono::steady_clock::now();
    tree_ms_ = std::chrono::duration<double, std::milli>(tt1 - tt0).count();
    // the walk on the GPU unless a cutoff predicate (host code) takes part
    if (plan_only || cutoff || !plan_.build_lists_gpu())
        plan_.build_lists(cutoff);
    lists_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tt1)
                    .count();
    const auto tt2 = std::chrono::steady_clock::now();
    plan_.assign_shards(shard_n_);
    // the target-leaf lists: on the host for a plan-only init, else built on
    // the GPU by setup_device
    if (plan_only)
        plan_.build_target_lists(shard_n_ > 1 ? shard_rank_ : -1);
    else
        plan_.collect_target_leaves();
    tlists_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tt2)
                     .count();
    if (tol_ > 0) // ifgfoperator.hpp:80-85
    {
        estimate_orders(base_order_);
        set_orders();
    }

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
            G.hfi[d] = 1.0 / G.hf[d];
            G.hci[d] = 1.0 / G.hc[d];
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
    const auto td = std::chrono::steady_clock::now();
    setup_device(normals);
    device_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - td)
                     .count();
    initialized_ = true;
    init_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

void Operator::setup_device(const double* normals)
{
    DeviceState& D = *dev_;
    // wall time of the setup phases (after a device synchronise), summed by name
    dev_phases_.clear();
    auto tp = std::chrono::steady_clock::now();
    auto phase = [&](const char* name) {
        IFGF_CUDA(cudaDeviceSynchronize());
        const auto now = std::chrono::steady_clock::now();
        const double ms = std::chrono::duration<double, std::milli>(now - tp).count();
        tp = now;
        for (auto& pr : dev_phases_)
            if (pr.first == name)
            {
                pr.second += ms;
                return;
            }
        dev_phases_.push_back({name, ms});
    };
    D.dgeo32.clear();
    D.dgeo32_ptr.clear();
    D.dgeo_ready = false;
    // the device this operator's tables live on
    IFGF_CUDA(cudaGetDevice(&device_));
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
        D.A_host = A;
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
        D.n_tleaf = (int)ntl;
    }
    phase("boxes_points_upload");
    build_target_lists_gpu(plan_, shard_n_ > 1 ? shard_rank_ : -1, D.tl_far_off, D.tl_far_src,
                           D.tl_near_off, D.tl_near_src);
    // the far-field plan of earlier tables is stale: rebuilt on first use
    D.fp_chunk.release();
    D.fp_group.release();
    D.fp_rec.release();
    D.fp_slot.release();
    D.fp_nchunk = 0;
    D.fp_ready = false;
    phase("target_leaf_lists");
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
    D.leaf_idx.clear();
    D.up_idx.clear();
    D.up_slot.clear();
    D.geo64.clear();
    D.geo32.clear();
    D.leaf_idx.resize(L);
    D.up_idx.resize(L);
    D.up_slot.resize(L);
    D.tc_runs.assign(L, {});
    D.tc_img.clear();
    D.tc_img_off.clear();
    D.tc_img_ready = false;
    D.tc_tiles.clear();
    D.tc_tiles.resize(L);
    D.tc_fill.assign(L, {});
    D.up_choice.clear();
    D.up_ms_ffma.clear();
    D.up_ms_tc.clear();
    D.geo64.resize(L);
    D.geo32.resize(L);
    D.fe_list.resize(L);
    D.slot_el.resize(L);
    D.child_off.resize(L);
    D.up_pH.assign(L, 0.0);
    D.up_cH.assign(L, 0.0);
    D.vkind = -1;
    D.vgeo64.clear();
    D.vgeo32.clear();
    D.vlists.clear();
    std::vector<std::vector<int>> up_host(L);
    phase("cone_map_alloc");
    // coarse cones each level refines: all of them, or this rank's
    const bool sharded = shard_n_ > 1;
    std::vector<std::vector<int>> c2f_host(L);
    D.c2f_idx.resize(L);
    std::vector<int> up_pad(L, 0);
    fe_pad_.assign(L, 0);
    up_stats_.assign(L, UpwardLevelStats{});
    upgeo_bytes_ = 0;
    int64_t coarse_tot = 0, fine_tot = 0;
    leaf_evals_ = upward_evals_ = 0;
    // point range of every target box, by global id, for the far pairs of
    // the cone-marking kernel (read from the device pair lists)
    DevBuf<int> tbox_first, tbox_last;
    {
        std::vector<int> tf, tl;
        plan_.target_box_ranges(tf, tl);
        tbox_first.upload(tf);
        tbox_last.upload(tl);
    }
    plan_.ensure_device_pairs();
    for (int l = 0; l < L; l++)
    {
        LevelGeom& G = lv_[l];
        const int64_t nce = (int64_t)G.nc[0] * G.nc[1] * G.nc[2];
        const int64_t nfe = (int64_t)G.nf[0] * G.nf[1] * G.nf[2];
        const int64_t ncm = (int64_t)G.nbox * nce, nfm = (int64_t)G.nbox * nfe;
        IFGF_CUDA(cudaMemset(cmark.p, 0, ncm * sizeof(int)));
        phase("cone_marks");
        // far pairs of this level's source boxes: a contiguous range of the
        // source-major device pair list
        const int64_t p0 = plan_.far.off.empty() ? 0 : plan_.far.off[S.level_off[l]];
        const int64_t p1 = plan_.far.off.empty() ? 0 : plan_.far.off[S.level_off[l + 1]];
        if (p1 > p0)
        {
            mark_far_kernel<<<(unsigned)(p1 - p0), 128>>>(
                G, TA, plan_.far_dev.src.get() + p0, plan_.far_dev.tgt.get() + p0, tbox_first.p,
                tbox_last.p, D.tx.p, D.ty.p, D.tz.p, D.fmap.p, cmark.p);
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
        phase("mark_far_parent_kernels");
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
        phase("compaction");
        // leaf / non-leaf partition of the coarse cones and the work counts
        // of the flop model
        std::vector<int> lidx, uidx;
        if (G.n_coarse > 0)
        {
            std::vector<int> cb(G.n_coarse);
            IFGF_CUDA(cudaMemcpy(cb.data(), D.cc_box[l].p, cb.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < G.n_coarse; i++)
            {
                const int g = cb[i];
                if (sharded && plan_.box_rank[g] != shard_rank_)
                    continue; // another rank's subtree
                c2f_host[l].push_back((int)i);
                if (bleaf[g])
                {
                    lidx.push_back((int)i);
                    leaf_evals_ += (double)P_hi * (bl[g] - bf[g]);
                }
                else
                {
                    uidx.push_back((int)i);
                    int nch = 0;
                    for (int j = 0; j < 8; j++)
                        nch += bch[8 * g + j] >= 0;
                    upward_evals_ += (double)P_hi * nch;
                }
            }
        }
        D.leaf_idx[l].upload(lidx);
        up_host[l] = std::move(uidx);
        phase("cone_partition_host");
    }
    // Upward transfer: order each level's cones of non-leaf boxes by element
    // (stable, so boxes stay ordered within an element), give every distinct
    // element a slot and tabulate the box-independent geometry per slot.
    for (int l = 0; l + 1 < L; l++)
    {
        std::vector<int>& uidx = up_host[l];
        std::vector<int> slot_of(uidx.size()), slot_el;
        if (!uidx.empty())
        {
            std::vector<int> el(lv_[l].n_coarse);
            IFGF_CUDA(cudaMemcpy(el.data(), D.cc_el[l].p, el.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost));
            stable_order_by_key(uidx, el);
            for (size_t i = 0; i < uidx.size(); i++)
            {
                if (i == 0 || el[uidx[i]] != el[uidx[i - 1]])
                    slot_el.push_back(el[uidx[i]]);
                slot_of[i] = (int)slot_el.size() - 1;
            }
            // child-centre offsets of a box of this level, as the tree builds them
            const TreeLevel& TL = S.levels[l];
            double off[24];
            for (int o = 0; o < 8; o++)
                for (int d = 0; d < 3; d++)
                {
                    const double mn = TL.bbmin[d], mx = TL.bbmax[d];
                    const double size = 0.5 * (mx - mn);
                    const double cmn = mn + size * (double)((o >> d) & 1), cmx = cmn + size;
                    off[3 * o + d] = (cmx + cmn) / 2.0 - (mx + mn) / 2.0;
                }
            DevBuf<double>& doff = D.child_off[l];
            doff.upload(off, 24);
            DevBuf<int>& dslot_el = D.slot_el[l];
            dslot_el.upload(slot_el);
            const KParams kp = make_kparams(kr_, ki_, dx_);
            const double pH = S.levels[l].side, cH = S.levels[l + 1].side;
            D.up_pH[l] = pH;
            D.up_cH[l] = cH;
            const int ns = (int)slot_el.size();
            DevBuf<int> drow;
            drow.alloc((size_t)ns * 16);
            std::vector<int> hrow((size_t)ns * 16);
            int pad = 0, runs = 0;
            phase("upward_slots_host");
            IFGF_DISPATCH(kind_, pad = upgeo_row_max<KK>(lv_[l], lv_[l + 1], pH, cH, doff.p,
                                                          dslot_el.p, ns, D.hi_nodes.p, P_hi, kp,
                                                          drow.p, hrow.data(), &runs));
            phase("upward_row_measure");
            up_pad[l] = pad;
            fe_pad_[l] = runs;
            {
                // work of this level's upward transfer: node evaluations,
                // child coefficient blocks (runs) and padded table entries
                UpwardLevelStats& us = up_stats_[l];
                us.cones = (int64_t)uidx.size();
                us.slots = ns;
                std::vector<int> cbox(lv_[l].n_coarse);
                IFGF_CUDA(cudaMemcpy(cbox.data(), D.cc_box[l].p, cbox.size() * sizeof(int),
                                     cudaMemcpyDeviceToHost));
                for (size_t i = 0; i < uidx.size(); i++)
                {
                    const int g = cbox[uidx[i]];
                    for (int o = 0; o < 8; o++)
                        if (bch[8 * g + o] >= 0)
                        {
                            us.blocks += hrow[2 * ((size_t)slot_of[i] * 8 + o) + 1];
                            us.entries += hrow[2 * ((size_t)slot_of[i] * 8 + o)];
                        }
                }
            }
            phase("upward_stats_host");
            D.fe_list[l].alloc((size_t)ns * 8 * (runs + 1)); // runs and a sentinel per row
            IFGF_CUDA(cudaMemset(D.fe_list[l].p, 0xff, D.fe_list[l].n * sizeof(int2)));
            const size_t n_ent = (size_t)ns * 8 * (size_t)std::max(pad, 1);
            D.geo64[l].alloc(n_ent);
            D.geo32[l].alloc(n_ent);
            // all-ones bytes: element -1 and node -1 mark skipped entries
            IFGF_CUDA(cudaMemset(D.geo64[l].p, 0xff, n_ent * sizeof(UpGeo64)));
            IFGF_CUDA(cudaMemset(D.geo32[l].p, 0xff, n_ent * sizeof(UpGeo32)));
            IFGF_DISPATCH(kind_, launch_build_upgeo<KK>(lv_[l], lv_[l + 1], pH, cH, doff.p,
                                                         dslot_el.p, ns, D.hi_nodes.p, P_hi, kp,
                                                         pad, D.geo64[l].p, D.geo32[l].p, runs,
                                                         D.fe_list[l].p));
            IFGF_CUDA(cudaDeviceSynchronize());
            upgeo_bytes_ += (double)n_ent * (sizeof(UpGeo64) + sizeof(UpGeo32));
            phase("upward_table_build");
        }
        D.up_idx[l].upload(uidx);
        D.up_slot[l].upload(slot_of);
        // runs of equal slots (first position, cones): the tensor-core
        // kernel's tiles never mix slots
        std::vector<int2>& runs = D.tc_runs[l];
        runs.clear();
        for (size_t i = 0; i < slot_of.size(); i++)
            if (i == 0 || slot_of[i] != slot_of[i - 1])
                runs.push_back(make_int2((int)i, 1));
            else
                runs.back().y++;
    }
    phase("upward_uploads");
    D.lists.assign(L, LevelLists{});
    for (int l = 0; l < L; l++)
    {
        if (sharded)
            D.c2f_idx[l].upload(c2f_host[l]);
        D.lists[l] = LevelLists{D.cc_box[l].p, D.cc_el[l].p, D.leaf_idx[l].p, D.up_idx[l].p,
                                D.up_slot[l].p, D.geo64[l].p, D.geo32[l].p,
                                (int)D.leaf_idx[l].n, (int)D.up_idx[l].n, up_pad[l],
                                D.fe_list[l].p, fe_pad_[l],
                                sharded ? D.c2f_idx[l].p : nullptr,
                                sharded ? (int)c2f_host[l].size() : -1};
    }
    // single-plane tiles of the tensor-core upward transfer (built here, so
    // that a matvec never allocates them)
    ensure_tc_tiles(1);
    for (int l = 0; l < L; l++)
    {
        D.lists[l].tc_tiles = D.tc_tiles[l][1].p;
        D.lists[l].n_tc_tiles = (int)D.tc_tiles[l][1].n;
        D.lists[l].tc_fill = D.tc_fill[l][1];
    }
    D.tc_status.alloc(1);
    D.tc_status.zero();
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
    D.unear.alloc(Tt.n);
    D.err.alloc(1);
    D.err.zero();
    if (!D.side)
        IFGF_CUDA(cudaStreamCreateWithFlags(&D.side, cudaStreamNonBlocking));
    if (!D.ev_fork)
        IFGF_CUDA(cudaEventCreateWithFlags(&D.ev_fork, cudaEventDisableTiming));
    if (!D.ev_join)
        IFGF_CUDA(cudaEventCreateWithFlags(&D.ev_join, cudaEventDisableTiming));
    const int F0 = fct_[0] * lo_[0], F1 = fct_[1] * lo_[1];
    const size_t sz2 = std::max<size_t>((size_t)F0 * hi_[1] * hi_[2], (size_t)F0 * F1 * lo_[2]);
    D.c2f_smem = (P_hi + sz2 + (size_t)F0 * F1 * hi_[2]) * sizeof(double2);
    if (D.c2f_smem > 220 * 1024)
        throw Error(ERR_INVALID, "interpolation order too high for the coarse-to-fine kernel");
    phase("buffers");
}

// CUDA-event timing of every launch, used when profiling is on.
struct EventHooks : LaunchHooks
{
    DeviceState& D;
    cudaStream_t st;
    std::vector<int> cls;
    int n = 0;
    EventHooks(DeviceState& d, cudaStream_t s) : D(d), st(s) {}
    std::vector<int> lev;
    void begin(int c, int level) override
    {
        lev.push_back(level);
        while ((int)D.prof_ev.size() < 2 * (n + 1))
        {
            cudaEvent_t e;
            IFGF_CUDA(cudaEventCreate(&e));
            D.prof_ev.push_back(e);
        }
        cls.push_back(c);
        IFGF_CUDA(cudaEventRecord(D.prof_ev[2 * n], st));
    }
    void end() override
    {
        IFGF_CUDA(cudaEventRecord(D.prof_ev[2 * n + 1], st));
        n++;
    }
};

void Operator::fill_mult_ptrs(MultPtrs& m, bool variant) const
{
    const DeviceState& D = *dev_;
    m.L = (int)lv_.size();
    m.lv_host = lv_.data();
    m.lv_dev = D.lv.p;
    m.lists = variant ? D.vlists.data() : D.lists.data();
    m.T = TreeArgs{D.box_c.p, D.box_H.p, D.box_first.p, D.box_last.p, D.box_child.p,
                   D.box_level.p, D.box_leaf.p};
    m.S = SrcArgs{D.sx.p, D.sy.p, D.sz.p, D.nx.p, D.ny.p, D.nz.p};
    m.tx = D.tx.p;
    m.ty = D.ty.p;
    m.tz = D.tz.p;
    m.src_perm = D.src_perm.p;
    m.tgt_perm = D.tgt_perm.p;
    m.hi_nodes = D.hi_nodes.p;
    m.A = D.A.p;
    m.A_host = D.A_host.data();
    m.fmap = D.fmap.p;
    m.tl_first = D.tl_first.p;
    m.tl_last = D.tl_last.p;
    m.tl_far_off = D.tl_far_off.p;
    m.tl_far_src = D.tl_far_src.p;
    m.tl_near_off = D.tl_near_off.p;
    m.tl_near_src = D.tl_near_src.p;
    m.n_tleaf = D.n_tleaf;
    m.n_src = (long long)D.w.n;
    m.w = D.w.p;
    m.cvals = D.cvals.p;
    m.fcoef = D.fcoef.p;
    m.unear = D.unear.p;
    m.err = D.err.p;
    m.side = D.side;
    m.ev_fork = D.ev_fork;
    m.ev_join = D.ev_join;
    for (int d = 0; d < 3; d++)
    {
        m.lo[d] = lo_[d];
        m.hi[d] = hi_[d];
        m.fct[d] = fct_[d];
    }
    m.P_lo = lo_[0] * lo_[1] * lo_[2];
    m.P_hi = hi_[0] * hi_[1] * hi_[2];
    m.c2f_smem = D.c2f_smem;
    m.kp = make_kparams(kr_, ki_, dx_);
    m.mixed = precision_ == PREC_MIXED;
    m.up_path = up_path_;
    m.tc_status = D.tc_status.p;
    auto it = D.up_choice.find(1);
    m.up_choice = it != D.up_choice.end() ? it->second.data() : nullptr;
}

// Runs the upward-kernel autotuner for launches over `planes` planes once
// (AUTO path, mixed precision): times the FFMA and the tensor-core kernel of
// every level on this operator's tables and buffers (bp: the batch planes;
// null: the single-plane buffers) and keeps the per-level choice.  It
// synchronises `st` once; the buffers it ran on are rewritten by the matvec
// that follows.
void Operator::ensure_tc_images()
{
    DeviceState& D = *dev_;
    if (D.tc_img_ready)
        return;
    D.tc_img_ready = true;
    const int L = (int)lv_.size();
    D.tc_img.resize(L);
    D.tc_img_off.resize(L);
    // levels whose slots have many cones (so many row tiles reuse every
    // image), most cones per slot first, within a memory budget
    std::vector<std::pair<double, int>> cand;
    for (int l = 0; l + 1 < L; l++)
    {
        const LevelLists& LL = D.lists[l];
        const int ns = (int)D.slot_el[l].n;
        if (LL.n_up <= 0 || ns == 0 || LL.up_pad <= 0 || LL.fe_pad <= 0)
            continue;
        const double cps = (double)LL.n_up / ns;
        if (cps >= UPTC_IMG_MIN_CONES)
            cand.push_back({cps, l});
    }
    std::sort(cand.begin(), cand.end(), [](auto& x, auto& y) { return x.first > y.first; });
    long long used = 0;
    for (const auto& c : cand)
    {
        const int l = c.second;
        LevelLists& LL = D.lists[l];
        const int ns = (int)D.slot_el[l].n;
        DevBuf<long long> sz;
        sz.alloc((size_t)ns * 8);
        if (!upward_tc_image_sizes(lo_, LL.fe_list, LL.fe_pad, LL.up_pad, ns, sz.p))
            return; // no tensor-core kernel for this order shape
        const std::vector<long long> hs = sz.download();
        std::vector<long long> off(hs.size());
        long long tot = 0;
        for (size_t i = 0; i < hs.size(); i++)
        {
            off[i] = tot;
            tot += hs[i];
        }
        if (tot == 0 || used + tot > UPTC_IMG_BUDGET)
            continue;
        D.tc_img_off[l].upload(off);
        D.tc_img[l].alloc((size_t)tot);
        upward_tc_image_fill(lo_, LL.fe_list, LL.fe_pad, LL.geo32, LL.up_pad, ns,
                             D.tc_img_off[l].p, D.tc_img[l].p);
        LL.tc_img = D.tc_img[l].p;
        LL.tc_img_off = D.tc_img_off[l].p;
        used += tot;
    }
}

void Operator::ensure_upward_tuned(int planes, const BatchPtrs* bp, void* stream)
{
    DeviceState& D = *dev_;
    if (up_path_ != UP_AUTO || precision_ != PREC_MIXED || D.up_choice.count(planes))
        return;
    const int L = (int)lv_.size();
    std::vector<signed char> ch(L, -1);
    std::vector<double> mf(L, 0.0), mt(L, 0.0);
    MultPtrs m;
    fill_mult_ptrs(m);
    IFGF_DISPATCH(kind_, tune_upward_kernels<KK>(m, bp, planes, (cudaStream_t)stream, ch.data(),
                                                 mf.data(), mt.data()));
    D.up_choice[planes] = std::move(ch);
    D.up_ms_ffma[planes] = std::move(mf);
    D.up_ms_tc[planes] = std::move(mt);
}

// Row tiles of the tensor-core upward transfer for launches over `planes`
// right-hand-side planes, per level: each run of cones of one slot in
// chunks of up to 32 / planes cones (planes <= 32) x min(planes, 32) planes.
void Operator::ensure_tc_tiles(int planes)
{
    DeviceState& D = *dev_;
    const int L = (int)lv_.size();
    const int pq = std::min(planes, 32), cpt = 32 / pq;
    for (int l = 0; l < L && l < (int)D.tc_runs.size(); l++)
    {
        if (D.tc_tiles[l].count(planes))
            continue;
        std::vector<int4> t;
        int64_t rows = 0;
        for (const int2& r : D.tc_runs[l])
            for (int cs = 0; cs < r.y; cs += cpt)
                for (int q0 = 0; q0 < planes; q0 += pq)
                {
                    const int nc = std::min(cpt, r.y - cs), nq = std::min(pq, planes - q0);
                    t.push_back(make_int4(r.x + cs, nc, q0, nq));
                    rows += (int64_t)nc * nq;
                }
        DevBuf<int4>& b = D.tc_tiles[l][planes];
        if (!t.empty())
            b.upload(t);
        D.tc_fill[l][planes] = t.empty() ? 0.f : (float)((double)rows / (32.0 * (double)t.size()));
    }
}

// The tensor-core tiles for a batch launch over bp.groups * BATCH_NB planes,
// and (single-wavenumber batches) the autotuner's choice for them.
void Operator::set_far_plan(bool on)
{
    far_plan_on_ = on;
    if (!on && dev_)
    {
        DeviceState& D = *dev_;
        D.fp_chunk.release();
        D.fp_group.release();
        D.fp_rec.release();
        D.fp_slot.release();
        D.fp_nchunk = 0;
        D.fp_ready = false;
    }
}

void Operator::ensure_far_plan()
{
    DeviceState& D = *dev_;
    if (D.fp_ready || !far_plan_on_ || D.n_tleaf == 0)
        return;
    const auto t0 = std::chrono::steady_clock::now();
    IFGF_CUDA(cudaSetDevice(device_));
    // chunks of up to 256 targets of every target leaf
    const std::vector<int> tf = D.tl_first.download(), tlast = D.tl_last.download();
    std::vector<int> c_leaf, c_t0, c_cnt;
    for (int i = 0; i < D.n_tleaf; i++)
        for (int t = tf[i]; t < tlast[i]; t += 256)
        {
            c_leaf.push_back(i);
            c_t0.push_back(t);
            c_cnt.push_back(std::min(256, tlast[i] - t));
        }
    const int nc = (int)c_leaf.size();
    if (nc == 0)
        return;
    DevBuf<int> d_leaf, d_t0, d_cnt;
    d_leaf.upload(c_leaf);
    d_t0.upload(c_t0);
    d_cnt.upload(c_cnt);
    DevBuf<long long> n_group, n_rec, n_slot, n_ovf;
    n_group.alloc(nc);
    n_rec.alloc(nc);
    n_slot.alloc(nc);
    n_ovf.alloc(nc);
    FarBuildArgs b{};
    b.lv = D.lv.p;
    b.L = (int)lv_.size();
    b.box_c = D.box_c.p;
    b.box_H = D.box_H.p;
    b.box_level = D.box_level.p;
    b.tx = D.tx.p;
    b.ty = D.ty.p;
    b.tz = D.tz.p;
    b.fmap = D.fmap.p;
    b.far_off = D.tl_far_off.p;
    b.far_src = D.tl_far_src.p;
    b.c_leaf = d_leaf.p;
    b.c_t0 = d_t0.p;
    b.c_cnt = d_cnt.p;
    b.err = D.err.p;
    b.n_group = n_group.p;
    b.n_rec = n_rec.p;
    b.n_slot = n_slot.p;
    b.n_ovf = n_ovf.p;
    // a smaller slot count where it lets more far CTAs reside per SM and at
    // most 3 % of the records would overflow it and read global memory
    // (measured at p = 9, slots holding the most-used cones: at N = 1e6,
    // k = 100, 16 slots and three CTAs faster than 24 with 2.2 %
    // overflowing, 18 faster still with 1.7 %; at N = 2e5 16 slots 4 %
    // slower with 6.4 %, 18 slots 2.6 % slower)
    auto count = [&](int nslot) {
        b.nslot = nslot;
        far_plan_build_kernel<false><<<nc, 256>>>(b);
        IFGF_CUDA(cudaGetLastError());
        IFGF_CUDA(cudaDeviceSynchronize());
    };
    {
        // the larger of the two smaller slot counts that still gives more
        // CTAs per SM than FAR_PLAN_SLOTS (fewer records overflow with more
        // slots); FAR_PLAN_SLOTS where neither does
        const int p_lo = lo_[0] * lo_[1] * lo_[2];
        const int full = far_plan_ctas(FAR_PLAN_SLOTS, p_lo, BATCH_NB);
        const int few = far_plan_ctas(FAR_PLAN_SLOTS_MID, p_lo, BATCH_NB) > full ? FAR_PLAN_SLOTS_MID
                        : far_plan_ctas(FAR_PLAN_SLOTS_FEW, p_lo, BATCH_NB) > full
                            ? FAR_PLAN_SLOTS_FEW
                            : FAR_PLAN_SLOTS;
        count(few);
        const std::vector<long long> ho = n_ovf.download(), hr0 = n_rec.download();
        long long o = 0, r = 0;
        for (int c = 0; c < nc; c++)
        {
            o += ho[c];
            r += hr0[c];
        }
        D.fp_ovf_few = r > 0 ? (double)o / (double)r : 0.0;
        if (few != FAR_PLAN_SLOTS && o * 100 > 3 * r)
            count(FAR_PLAN_SLOTS);
    }
    const std::vector<long long> hg = n_group.download(), hr = n_rec.download(),
                                 hs = n_slot.download();
    std::vector<long long> g_off(nc), r_off(nc), s_off(nc);
    long long tg = 0, tr = 0, ts = 0;
    std::vector<FarChunk> chunks(nc);
    for (int c = 0; c < nc; c++)
    {
        g_off[c] = tg;
        r_off[c] = tr;
        s_off[c] = ts;
        chunks[c] = FarChunk{tg, tg + hg[c], c_t0[c], c_cnt[c]};
        tg += hg[c];
        tr += hr[c];
        ts += hs[c];
    }
    if (ts > (1ll << 31) - 1)
        throw Error(ERR_OOM, "far-field plan: slot list exceeds 2^31 entries");
    D.fp_group.alloc(std::max(tg, 1ll));
    D.fp_rec.alloc(std::max(tr, 1ll));
    D.fp_slot.alloc(std::max(ts, 1ll));
    D.fp_chunk.upload(chunks);
    DevBuf<long long> dg, dr, ds;
    dg.upload(g_off);
    dr.upload(r_off);
    ds.upload(s_off);
    b.g_off = dg.p;
    b.rec_off = dr.p;
    b.slot_off = ds.p;
    b.group = D.fp_group.p;
    b.rec = D.fp_rec.p;
    b.slot = D.fp_slot.p;
    far_plan_build_kernel<true><<<nc, 256>>>(b);
    IFGF_CUDA(cudaGetLastError());
    IFGF_CUDA(cudaDeviceSynchronize());
    {
        // every chunk must end where the next one starts
        const std::vector<long long> eg = n_group.download(), er = n_rec.download(),
                                     es = n_slot.download();
        for (int c = 0; c < nc; c++)
            if (eg[c] != g_off[c] + hg[c] || er[c] != r_off[c] + hr[c] || es[c] != s_off[c] + hs[c])
            {
                D.fp_chunk.release();
                D.fp_group.release();
                D.fp_rec.release();
                D.fp_slot.release();
                throw Error(ERR_STATE, "far-field plan: the filling pass disagrees with the "
                                       "counting pass");
            }
    }
    D.fp_nchunk = nc;
    D.fp_nslot = b.nslot;
    D.fp_ready = true;
    D.fp_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                  .count();
}

void Operator::set_batch_far(BatchPtrs& bp)
{
    DeviceState& D = *dev_;
    ensure_far_plan();
    if (!D.fp_ready)
    {
        bp.fp_chunk = nullptr;
        return;
    }
    bp.fp_chunk = D.fp_chunk.p;
    bp.fp_nchunk = D.fp_nchunk;
    bp.fp_nslot = D.fp_nslot;
    bp.fp_group = D.fp_group.p;
    bp.fp_rec = D.fp_rec.p;
    bp.fp_slot = D.fp_slot.p;
}

void Operator::set_batch_tc(BatchPtrs& bp, void* stream)
{
    DeviceState& D = *dev_;
    if (!bp.kp_plane)
        ensure_tc_images();
    const int planes = bp.groups * BATCH_NB;
    ensure_tc_tiles(planes);
    const int L = (int)lv_.size();
    D.tcb_ptr.assign(L, nullptr);
    D.tcb_n.assign(L, 0);
    D.tcb_fill.assign(L, 0.f);
    for (int l = 0; l < L; l++)
    {
        const DevBuf<int4>& b = D.tc_tiles[l][planes];
        D.tcb_ptr[l] = b.p;
        D.tcb_n[l] = (int)b.n;
        D.tcb_fill[l] = D.tc_fill[l][planes];
    }
    bp.tc_tiles = D.tcb_ptr.data();
    bp.n_tc_tiles = D.tcb_n.data();
    bp.tc_fill = D.tcb_fill.data();
    bp.up_choice = nullptr;
    if (!bp.kp_plane)
    {
        ensure_upward_tuned(planes, &bp, stream);
        auto it = D.up_choice.find(planes);
        if (it != D.up_choice.end())
            bp.up_choice = it->second.data();
    }
}

// One thread waits on an mbarrier that nothing arrives at, bounded by
// limit_ns; out[0] = 1 when the wait gave up, out[1..2] = the nanoseconds it
// waited (low, high word).
static __global__ void bounded_wait_probe_kernel(unsigned long long limit_ns, unsigned* out)
{
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x != 0)
        return;
    tc::mbar_init(tc::smem_u32(&bar), 1);
    const unsigned long long t0 = tc::global_ns();
    const bool ok = tc::mbar_wait(tc::smem_u32(&bar), 0, limit_ns);
    const unsigned long long dt = tc::global_ns() - t0;
    out[0] = ok ? 0u : 1u;
    out[1] = (unsigned)(dt & 0xffffffffu);
    out[2] = (unsigned)(dt >> 32);
}

void bounded_wait_selftest(double limit_ms, double* waited_ms)
{
    if (!(limit_ms > 0) || limit_ms > 10000)
        throw Error(ERR_INVALID, "limit_ms must be in (0, 10000]");
    DevBuf<unsigned> out;
    out.alloc(3);
    out.zero();
    bounded_wait_probe_kernel<<<1, 32>>>((unsigned long long)(limit_ms * 1e6), out.p);
    IFGF_CUDA(cudaGetLastError());
    unsigned h[3];
    IFGF_CUDA(cudaMemcpy(h, out.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (waited_ms)
        *waited_ms = (double)(((unsigned long long)h[2] << 32) | h[1]) * 1e-6;
    if (h[0])
        throw Error(ERR_TIMEOUT, "bounded wait gave up after its limit (as designed)");
}

void Operator::set_upward_path(int path)
{
    if (path < UP_AUTO || path > UP_TENSOR)
        throw Error(ERR_INVALID, "upward path must be 0 (auto), 1 (FFMA) or 2 (tensor cores)");
    up_path_ = path;
}

// Reports a bounded device wait of a tensor-core kernel that gave up (the
// status word is cleared, so that the next call starts clean).
void Operator::check_device_status()
{
    DeviceState& D = *dev_;
    if (!D.tc_status.p)
        return;
    unsigned st = 0;
    IFGF_CUDA(cudaMemcpy(&st, D.tc_status.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (st)
    {
        IFGF_CUDA(cudaMemset(D.tc_status.p, 0, sizeof(unsigned)));
        throw Error(ERR_TIMEOUT, "a tensor-core kernel's bounded wait gave up (pipeline stalled); "
                                 "results of the last matvec are invalid");
    }
}


// ---------------------------------------------------------------------------
// Adjoint
// ---------------------------------------------------------------------------

// out = sign conj(in)
static __global__ void adj_conj_kernel(const double2* __restrict__ in, double2* out, long long n,
                                       double sign)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
    {
        const double2 v = in[i];
        out[i] = make_double2(sign * v.x, -sign * v.y);
    }
}

// out = sign conj(sum_d n_d z_d - i kap y)   (y may be null)
static __global__ void adj_combine_kernel(const double2* __restrict__ z0,
                                          const double2* __restrict__ z1,
                                          const double2* __restrict__ z2,
                                          const double2* __restrict__ y,
                                          const double* __restrict__ nx,
                                          const double* __restrict__ ny,
                                          const double* __restrict__ nz, double kap, double sign,
                                          double2* out, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
    {
        const double a = nx[i], b = ny[i], c = nz[i];
        double sr = a * z0[i].x + b * z1[i].x + c * z2[i].x;
        double si = a * z0[i].y + b * z1[i].y + c * z2[i].y;
        if (y)
        {
            sr += kap * y[i].y;
            si -= kap * y[i].x;
        }
        out[i] = make_double2(sign * sr, -sign * si);
    }
}

static unsigned elementwise_grid(long long n)
{
    return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16));
}

void Operator::ensure_adjoint()
{
    if (adj_)
        return;
    if (!initialized_)
        throw Error(ERR_STATE, "adjoint called before init");
    auto A = std::make_unique<AdjointState>();
    const int64_t ns = n_src(), nt = n_tgt();
    const bool sym = kind_ == K_LAPLACE || kind_ == K_HELMHOLTZ || kind_ == K_MODHELMHOLTZ;
    // an operator of kernel `kind` (wavenumber kr + i ki, component dx) from
    // the targets to the sources
    auto swapped = [&](int kind, double kr, double ki, int dx) {
        std::unique_ptr<Operator> op(
            new Operator(kind, kr, ki, leaf_, order0_, base_n_[0], tol_));
        op->set_dx(dx);
        op->set_precision(precision_);
        op->init(tgt_pts_.data(), nt, src_pts_.data(), ns, nullptr, cutoff_);
        return op;
    };
    if (sym && same_points_)
        A->mode = 0;
    else if (sym || kind_ == K_GRADHELMHOLTZ)
    {
        A->mode = 1;
        A->sign = kind_ == K_GRADHELMHOLTZ ? -1.0 : 1.0; // the gradient kernel is odd
        A->ops.push_back(swapped(kind_, kr_, ki_, dx_));
    }
    else if (kind_ == K_DOUBLELAYER)
    {
        // G_DL(x, n_s) = sum_d n_s[d] G_grad,d(x) with the same k
        A->mode = 2;
        A->sign = -1.0;
        for (int d = 0; d < 3; d++)
            A->ops.push_back(swapped(K_GRADHELMHOLTZ, kr_, ki_, d));
    }
    else if (kind_ == K_COMBINEDFIELD)
    {
        // G_CF = dG/dn_s - i kap G with G = e^{i kap r}/(4 pi r), and
        // dG/dn_s = -sum_d n_s[d] G_grad,d for the gradient kernel at k = -i kap
        A->mode = 3;
        A->sign = 1.0;
        for (int d = 0; d < 3; d++)
            A->ops.push_back(swapped(K_GRADHELMHOLTZ, 0.0, -kr_, d));
        A->ops.push_back(swapped(K_HELMHOLTZ, kr_, 0.0, -1));
    }
    else
        throw Error(ERR_INVALID, "no adjoint for this kernel");
    if (!is_real())
        A->wc.alloc(nt);
    for (size_t i = 0; i < A->ops.size() || (A->mode == 0 && i == 0); i++)
        if (!is_real())
            A->z[i].alloc(ns);
    if (A->mode >= 2)
    {
        if (normals_.size() != (size_t)(3 * ns))
            throw Error(ERR_STATE, "the adjoint of this kernel needs the source normals");
        std::vector<double> c(ns);
        DevBuf<double>* dst[3] = {&A->nx, &A->ny, &A->nz};
        for (int d = 0; d < 3; d++)
        {
            for (int64_t i = 0; i < ns; i++)
                c[i] = normals_[3 * i + d];
            dst[d]->upload(c);
        }
    }
    adj_ = std::move(A);
}

void Operator::mult_adjoint_device(const void* d_w, void* d_u, void* stream)
{
    if (!d_w || !d_u)
        throw Error(ERR_INVALID, "null density or result buffer");
    ensure_adjoint();
    AdjointState& A = *adj_;
    cudaStream_t st = (cudaStream_t)stream;
    const long long ns = n_src(), nt = n_tgt();
    if (is_real())
    {
        // A^H = A^T for the real Laplace kernel
        if (A.mode == 0)
            mult_device(d_w, d_u, stream);
        else
            A.ops[0]->mult_device(d_w, d_u, stream);
        return;
    }
    adj_conj_kernel<<<elementwise_grid(nt), 256, 0, st>>>((const double2*)d_w, A.wc.p, nt, 1.0);
    IFGF_CUDA(cudaGetLastError());
    double2* u = (double2*)d_u;
    switch (A.mode)
    {
    case 0:
        mult_device(A.wc.p, A.z[0].p, stream);
        adj_conj_kernel<<<elementwise_grid(ns), 256, 0, st>>>(A.z[0].p, u, ns, A.sign);
        break;
    case 1:
        A.ops[0]->mult_device(A.wc.p, A.z[0].p, stream);
        adj_conj_kernel<<<elementwise_grid(ns), 256, 0, st>>>(A.z[0].p, u, ns, A.sign);
        break;
    default:
        for (size_t i = 0; i < A.ops.size(); i++)
            A.ops[i]->mult_device(A.wc.p, A.z[i].p, stream);
        adj_combine_kernel<<<elementwise_grid(ns), 256, 0, st>>>(
            A.z[0].p, A.z[1].p, A.z[2].p, A.mode == 3 ? A.z[3].p : nullptr, A.nx.p, A.ny.p,
            A.nz.p, kr_, A.sign, u, ns);
        break;
    }
    IFGF_CUDA(cudaGetLastError());
}

void Operator::mult_adjoint_host(const void* w, void* u, int64_t batch)
{
    if (!initialized_)
        throw Error(ERR_STATE, "adjoint called before init");
    if (!w || !u)
        throw Error(ERR_INVALID, "null density or result buffer");
    if (batch < 1)
        throw Error(ERR_INVALID, "batch must be >= 1");
    ensure_adjoint();
    AdjointState& A = *adj_;
    const size_t per = is_real() ? 1 : 2;
    const size_t nw = per * (size_t)n_tgt(), nu = per * (size_t)n_src();
    if (A.io_w.n < nw)
        A.io_w.alloc(nw);
    if (A.io_u.n < nu)
        A.io_u.alloc(nu);
    for (int64_t b = 0; b < batch; b++)
    {
        IFGF_CUDA(cudaMemcpy(A.io_w.p, (const double*)w + b * nw, nw * sizeof(double),
                             cudaMemcpyHostToDevice));
        mult_adjoint_device(A.io_w.p, A.io_u.p, nullptr);
        IFGF_CUDA(cudaMemcpy((double*)u + b * nu, A.io_u.p, nu * sizeof(double),
                             cudaMemcpyDeviceToHost));
    }
}

int Operator::dk_kind() const
{
    return kind_ == K_HELMHOLTZ ? K_HELMHOLTZ_DK : kind_ == K_COMBINEDFIELD ? K_COMBINEDFIELD_DK : -1;
}

// Upward geometry tables of another kernel on the same tree and cones: the
// rows (elements, nodes, local coordinates, runs) are the base kernel's and
// only the centre-shift factors differ, so the fill pass simply runs again
// with the variant kernel.
void Operator::ensure_variant_tables(int vkind)
{
    DeviceState& D = *dev_;
    if (D.vkind == vkind)
        return;
    const int L = (int)lv_.size();
    const int P_hi = hi_[0] * hi_[1] * hi_[2];
    const KParams kp = make_kparams(kr_, ki_, dx_);
    D.vkind = -1;
    D.vgeo64.clear();
    D.vgeo32.clear();
    D.vgeo64.resize(L);
    D.vgeo32.resize(L);
    D.vlists = D.lists;
    for (auto& VL : D.vlists) // the images hold the base kernel's centre-shift factors
    {
        VL.tc_img = nullptr;
        VL.tc_img_off = nullptr;
    }
    for (int l = 0; l + 1 < L; l++)
    {
        const LevelLists& LL = D.lists[l];
        const int ns = (int)D.slot_el[l].n;
        if (ns == 0 || LL.up_pad <= 0)
            continue;
        const size_t n_ent = (size_t)ns * 8 * (size_t)LL.up_pad;
        D.vgeo64[l].alloc(n_ent);
        D.vgeo32[l].alloc(n_ent);
        IFGF_CUDA(cudaMemset(D.vgeo64[l].p, 0xff, n_ent * sizeof(UpGeo64)));
        IFGF_CUDA(cudaMemset(D.vgeo32[l].p, 0xff, n_ent * sizeof(UpGeo32)));
        IFGF_DISPATCH(vkind, launch_build_upgeo<KK>(lv_[l], lv_[l + 1], D.up_pH[l], D.up_cH[l],
                                                     D.child_off[l].p, D.slot_el[l].p, ns,
                                                     D.hi_nodes.p, P_hi, kp, LL.up_pad,
                                                     D.vgeo64[l].p, D.vgeo32[l].p, LL.fe_pad,
                                                     D.fe_list[l].p));
        IFGF_CUDA(cudaDeviceSynchronize());
        D.vlists[l].geo64 = D.vgeo64[l].p;
        D.vlists[l].geo32 = D.vgeo32[l].p;
    }
    D.vkind = vkind;
}

void Operator::mult_dk_device(const void* d_w, void* d_u, void* stream)
{
    const int vk = dk_kind();
    if (vk < 0)
        throw Error(ERR_INVALID, "the k-derivative exists for the Helmholtz and combined-field "
                                 "kernels only");
    launch_mult(d_w, d_u, stream, false, vk);
}

void Operator::mult_dk_host(const void* w, void* u, int64_t batch)
{
    const int vk = dk_kind();
    if (vk < 0)
        throw Error(ERR_INVALID, "the k-derivative exists for the Helmholtz and combined-field "
                                 "kernels only");
    host_mult_loop(w, u, batch, vk);
}

void Operator::launch_mult(const void* d_w, void* d_u, void* stream, bool timed, int vkind)
{
    if (!initialized_)
        throw Error(ERR_STATE, "mult called before init");
    if (!d_w || !d_u)
        throw Error(ERR_INVALID, "null density or result buffer");
    cudaStream_t st = (cudaStream_t)stream;
    DeviceState& D = *dev_;
    if (vkind >= 0)
        ensure_variant_tables(vkind);
    if (vkind < 0 && precision_ == PREC_MIXED)
    {
        ensure_tc_images();
        ensure_upward_tuned(1, nullptr, stream);
    }
    MultPtrs m;
    fill_mult_ptrs(m, vkind >= 0);
    EventHooks log(D, st);
    const bool on = profiling_ || timed;
    int launches = 0;
    IFGF_DISPATCH(vkind >= 0 ? vkind : kind_,
                  launches = launch_mult_kernels<KK>(m, d_w, d_u, is_real(), st,
                                                     on ? &log : nullptr));
    launches_per_mult_ = launches;
    if (on && log.n > 0)
        finish_profile(log, 1);
}

// Per-kernel times of the launches recorded in `log` (one matvec, or one
// batched group of `rhs` right-hand sides).
void Operator::finish_profile(EventHooks& log, int rhs)
{
    DeviceState& D = *dev_;
    {
        IFGF_CUDA(cudaEventSynchronize(D.prof_ev[2 * log.n - 1]));
        double cls_ms[NPROF] = {};
        for (int i = 0; i < log.n; i++)
        {
            float ms = 0;
            IFGF_CUDA(cudaEventElapsedTime(&ms, D.prof_ev[2 * i], D.prof_ev[2 * i + 1]));
            cls_ms[log.cls[i]] += ms;
            if (profiling_)
            {
                prof_ms_[log.cls[i]] += ms;
                prof_launches_[log.cls[i]]++;
                if (log.lev[i] >= 0 && log.lev[i] < MAX_LEVELS)
                    prof_level_ms_[log.cls[i]][log.lev[i]] += ms;
            }
        }
        float tot = 0;
        IFGF_CUDA(cudaEventElapsedTime(&tot, D.prof_ev[0], D.prof_ev[2 * log.n - 1]));
        if (profiling_)
            mults_profiled_ += rhs;
        last_.permute = cls_ms[PROF_PERMUTE];
        last_.coarse = cls_ms[PROF_COARSE];
        last_.c2f = cls_ms[PROF_C2F];
        last_.eval = cls_ms[PROF_EVAL];
        last_.upward = cls_ms[PROF_UPWARD];
        last_.near = cls_ms[PROF_NEAR];
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
        for (int l = 0; l < MAX_LEVELS; l++)
            prof_level_ms_[i][l] = 0;
    }
    mults_profiled_ = 0;
}

void Operator::mult_device(const void* d_w, void* d_u, void* stream)
{
    launch_mult(d_w, d_u, stream, false);
}

void Operator::mult_host(const void* w, void* u, int64_t batch)
{
    if (batch > 1 && precision_ == PREC_MIXED)
    {
        // the batched device pipeline on staged copies of all right-hand sides
        DeviceState& D = *dev_;
        if (!w || !u)
            throw Error(ERR_INVALID, "null density or result buffer");
        const size_t per = is_real() ? 1 : 2;
        const size_t nw = per * (size_t)n_src() * batch, nu = per * (size_t)n_tgt() * batch;
        if (D.io_w.n < nw)
            D.io_w.alloc(nw);
        if (D.io_u.n < nu)
            D.io_u.alloc(nu);
        auto pinned = [](const void* p) {
            cudaPointerAttributes at;
            if (cudaPointerGetAttributes(&at, p) != cudaSuccess)
            {
                cudaGetLastError();
                return false;
            }
            return at.type == cudaMemoryTypeHost;
        };
        if (batch > BATCH_NB && pinned(w) && pinned(u))
        {
            // pinned host buffers: groups of BATCH_NB right-hand sides, the
            // next group's upload and the previous group's download overlap
            // this group's matvec
            for (cudaStream_t* st : {&D.io_cs, &D.io_up, &D.io_down})
                if (!*st)
                    IFGF_CUDA(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking));
            // a lone last right-hand side joins the group before it: every
            // group then runs the batched kernels, with planes grouped as in
            // a single call (same results)
            const int64_t ng = batch / BATCH_NB + (batch % BATCH_NB > 1 ? 1 : 0);
            auto group = [&](int64_t g, int64_t& b0, int64_t& cnt) {
                b0 = g * BATCH_NB;
                cnt = g + 1 < ng ? BATCH_NB : batch - b0;
            };
            while ((int64_t)D.io_ev.size() < 2 * ng)
            {
                cudaEvent_t e;
                IFGF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                D.io_ev.push_back(e);
            }
            const size_t pw = per * (size_t)n_src(), pu = per * (size_t)n_tgt();
            for (int64_t g = 0; g < ng; g++)
            {
                int64_t b0, cnt;
                group(g, b0, cnt);
                IFGF_CUDA(cudaMemcpyAsync(D.io_w.p + b0 * pw, (const double*)w + b0 * pw,
                                          cnt * pw * sizeof(double), cudaMemcpyHostToDevice,
                                          D.io_up));
                IFGF_CUDA(cudaEventRecord(D.io_ev[2 * g], D.io_up));
            }
            for (int64_t g = 0; g < ng; g++)
            {
                int64_t b0, cnt;
                group(g, b0, cnt);
                IFGF_CUDA(cudaStreamWaitEvent(D.io_cs, D.io_ev[2 * g], 0));
                mult_batch_device(D.io_w.p + b0 * pw, D.io_u.p + b0 * pu, cnt, D.io_cs);
                IFGF_CUDA(cudaEventRecord(D.io_ev[2 * g + 1], D.io_cs));
                IFGF_CUDA(cudaStreamWaitEvent(D.io_down, D.io_ev[2 * g + 1], 0));
                IFGF_CUDA(cudaMemcpyAsync((double*)u + b0 * pu, D.io_u.p + b0 * pu,
                                          cnt * pu * sizeof(double), cudaMemcpyDeviceToHost,
                                          D.io_down));
            }
            IFGF_CUDA(cudaStreamSynchronize(D.io_down));
            IFGF_CUDA(cudaStreamSynchronize(D.io_cs));
        }
        else
        {
            IFGF_CUDA(cudaMemcpy(D.io_w.p, w, nw * sizeof(double), cudaMemcpyHostToDevice));
            mult_batch_device(D.io_w.p, D.io_u.p, batch, nullptr);
            IFGF_CUDA(cudaMemcpy(u, D.io_u.p, nu * sizeof(double), cudaMemcpyDeviceToHost));
        }
        IFGF_CUDA(cudaMemcpy(&missing_, D.err.p, sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost));
        check_device_status();
        return;
    }
    host_mult_loop(w, u, batch, -1);
}

void Operator::mult_batch_device(const void* d_w, void* d_u, int64_t batch, void* stream)
{
    if (!initialized_)
        throw Error(ERR_STATE, "mult called before init");
    if (!d_w || !d_u)
        throw Error(ERR_INVALID, "null density or result buffer");
    if (batch < 1)
        throw Error(ERR_INVALID, "batch must be >= 1");
    DeviceState& D = *dev_;
    const size_t per = is_real() ? 1 : 2;
    const long long in_plane = (long long)(per * n_src()), out_plane = (long long)(per * n_tgt());
    int64_t done = 0;
    if (precision_ == PREC_MIXED && batch > 1)
    {
        const int planes = ensure_batch_planes(batch);
        BatchPtrs bp = batch_ptrs(in_plane, out_plane);
        set_batch_far(bp);
        MultPtrs m;
        fill_mult_ptrs(m);
        cudaStream_t st = (cudaStream_t)stream;
        while (done < batch)
        {
            bp.nrhs = (int)std::min<int64_t>(planes, batch - done);
            bp.groups = (bp.nrhs + BATCH_NB - 1) / BATCH_NB;
            set_batch_tc(bp, st);
            EventHooks log(D, st);
            int r = -1;
            IFGF_DISPATCH(kind_, r = launch_mult_batch_kernels<KK>(
                                     m, bp, (const double*)d_w + done * in_plane,
                                     (double*)d_u + done * out_plane, is_real(), st,
                                     profiling_ ? &log : nullptr));
            if (r < 0)
                break; // no batched path for this shape
            launches_per_mult_ = r;
            if (profiling_ && log.n > 0)
                finish_profile(log, bp.nrhs);
            done += bp.nrhs;
        }
    }
    for (; done < batch; done++)
        launch_mult((const double*)d_w + done * in_plane, (double*)d_u + done * out_plane, stream,
                    false);
}

// Plane buffers of the batched pipeline for up to `want` right-hand sides
// (whole groups of BATCH_NB, within a 16 GB budget and 64 planes), sized for
// the current tree; returns the planes one launch may use.
int Operator::ensure_batch_planes(int64_t want)
{
    DeviceState& D = *dev_;
    const size_t plane_bytes = sizeof(float2) * ((size_t)n_src() + D.cvals.n + D.fcoef.n) +
                               sizeof(double2) * (size_t)n_tgt();
    const int64_t budget = (int64_t)(16ull << 30) / (int64_t)std::max<size_t>(plane_bytes, 1);
    int cap = (int)std::min<int64_t>(64, budget) / BATCH_NB * BATCH_NB;
    cap = std::max(cap, BATCH_NB);
    const int planes =
        (int)std::min<int64_t>(cap, (want + BATCH_NB - 1) / BATCH_NB * BATCH_NB);
    if (D.b_planes >= planes && D.b_cv == D.cvals.n && D.b_fc == D.fcoef.n && D.b_ns == n_src() &&
        D.b_nt == n_tgt())
        return std::min(planes, D.b_planes);
    D.bw.alloc((size_t)planes * n_src());
    D.bcv.alloc((size_t)planes * D.cvals.n);
    D.bfc.alloc((size_t)planes * D.fcoef.n);
    D.bfc.zero(); // fine cones without an active coarse parent read zero
    D.bun.alloc((size_t)planes * n_tgt());
    D.b_planes = planes;
    D.b_cv = D.cvals.n;
    D.b_fc = D.fcoef.n;
    D.b_ns = n_src();
    D.b_nt = n_tgt();
    return planes;
}

BatchPtrs Operator::batch_ptrs(long long in_plane, long long out_plane) const
{
    const DeviceState& D = *dev_;
    BatchPtrs bp;
    bp.w = D.bw.p;
    bp.cvals = D.bcv.p;
    bp.fcoef = D.bfc.p;
    bp.unear = D.bun.p;
    bp.cv_plane = (long long)D.cvals.n;
    bp.fc_plane = (long long)D.fcoef.n;
    bp.n_src = n_src();
    bp.n_tgt = n_tgt();
    bp.in_plane = in_plane;
    bp.out_plane = out_plane;
    return bp;
}

// Distance tables of every level (UpGeo32 with tr = d - d_parent,
// ti = d_parent / d): the upward geometry of multi-wavenumber batches.
void Operator::ensure_distance_tables()
{
    DeviceState& D = *dev_;
    if (D.dgeo_ready)
        return;
    const int L = (int)lv_.size();
    const int P_hi = hi_[0] * hi_[1] * hi_[2];
    const KParams kp = make_kparams(kr_, ki_, dx_);
    D.dgeo32.clear();
    D.dgeo32.resize(L);
    D.dgeo32_ptr.assign(L, nullptr);
    for (int l = 0; l + 1 < L; l++)
    {
        const LevelLists& LL = D.lists[l];
        const int ns = (int)D.slot_el[l].n;
        if (ns == 0 || LL.up_pad <= 0)
            continue;
        const size_t n_ent = (size_t)ns * 8 * (size_t)LL.up_pad;
        D.dgeo32[l].alloc(n_ent);
        IFGF_CUDA(cudaMemset(D.dgeo32[l].p, 0xff, n_ent * sizeof(UpGeo32)));
        IFGF_DISPATCH(kind_, launch_build_upgeo<KK>(lv_[l], lv_[l + 1], D.up_pH[l], D.up_cH[l],
                                                     D.child_off[l].p, D.slot_el[l].p, ns,
                                                     D.hi_nodes.p, P_hi, kp, LL.up_pad, nullptr,
                                                     D.dgeo32[l].p, LL.fe_pad, D.fe_list[l].p));
        D.dgeo32_ptr[l] = D.dgeo32[l].p;
    }
    IFGF_CUDA(cudaDeviceSynchronize());
    D.dgeo_ready = true;
}

void Operator::mult_wavenumbers_host(const double* k, int64_t nk, const void* w, void* u)
{
    if (!initialized_)
        throw Error(ERR_STATE, "mult called before init");
    if (!w || !u)
        throw Error(ERR_INVALID, "null density or result buffer");
    if (nk < 1)
        throw Error(ERR_INVALID, "need at least one wavenumber");
    DeviceState& D = *dev_;
    const size_t per = is_real() ? 1 : 2;
    const size_t nw = per * (size_t)n_src() * nk, nu = per * (size_t)n_tgt() * nk;
    if (D.io_w.n < nw)
        D.io_w.alloc(nw);
    if (D.io_u.n < nu)
        D.io_u.alloc(nu);
    IFGF_CUDA(cudaMemcpy(D.io_w.p, w, nw * sizeof(double), cudaMemcpyHostToDevice));
    mult_wavenumbers_device(k, nk, D.io_w.p, D.io_u.p, nullptr);
    IFGF_CUDA(cudaMemcpy(u, D.io_u.p, nu * sizeof(double), cudaMemcpyDeviceToHost));
    IFGF_CUDA(cudaMemcpy(&missing_, D.err.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    check_device_status();
}

void Operator::mult_wavenumbers_device(const double* k, int64_t nk, const void* d_w, void* d_u,
                                       void* stream)
{
    if (!initialized_)
        throw Error(ERR_STATE, "mult called before init");
    if (!k || !d_w || !d_u)
        throw Error(ERR_INVALID, "null wavenumber, density or result buffer");
    if (nk < 1)
        throw Error(ERR_INVALID, "need at least one wavenumber");
    for (int64_t p = 0; p < nk; p++)
    {
        if (!std::isfinite(k[2 * p]) || !std::isfinite(k[2 * p + 1]))
            throw Error(ERR_INVALID, "wavenumber must be finite");
        if (!grids_match(k[2 * p], k[2 * p + 1]))
            throw Error(ERR_INVALID, "wavenumber " + std::to_string(k[2 * p]) + (k[2 * p + 1] < 0 ? "" : "+") +
                                         std::to_string(k[2 * p + 1]) +
                                         "i gives other cone grids than the operator's; "
                                         "use set_wavenumber for it");
    }
    DeviceState& D = *dev_;
    const size_t per = is_real() ? 1 : 2;
    const long long in_plane = (long long)(per * n_src()), out_plane = (long long)(per * n_tgt());
    cudaStream_t st = (cudaStream_t)stream;
    adj_.reset();
    if (precision_ != PREC_MIXED)
    {
        // FP64: the centre-shift factors of each wavenumber, then its matvec
        const double okr = kr_, oki = ki_;
        for (int64_t p = 0; p < nk; p++)
        {
            IFGF_CUDA(cudaStreamSynchronize(st)); // the tables are rebuilt in place
            set_wavenumber(k[2 * p], k[2 * p + 1]);
            launch_mult((const double*)d_w + p * in_plane, (double*)d_u + p * out_plane, stream,
                        false);
        }
        IFGF_CUDA(cudaStreamSynchronize(st));
        set_wavenumber(okr, oki);
        return;
    }
    ensure_distance_tables();
    const int planes = ensure_batch_planes(nk);
    // every plane's wavenumber, padded to whole groups
    const int64_t nk_pad = (nk + BATCH_NB - 1) / BATCH_NB * BATCH_NB;
    std::vector<KParams> kps((size_t)nk_pad);
    for (int64_t p = 0; p < nk_pad; p++)
    {
        const int64_t q = std::min(p, nk - 1);
        kps[(size_t)p] = make_kparams(k[2 * q], k[2 * q + 1], dx_);
    }
    // uploaded only when they change: a repeated call (the same frequency
    // set) then enqueues kernels only, so that it can be captured into a
    // CUDA graph after a first call
    bool same_k = D.kp_host.size() == kps.size();
    for (size_t i = 0; same_k && i < kps.size(); i++)
        same_k = D.kp_host[i].kr == kps[i].kr && D.kp_host[i].ki == kps[i].ki &&
                 D.kp_host[i].dx == kps[i].dx;
    if (!same_k)
    {
        if (D.kp_plane.n < kps.size())
            D.kp_plane.alloc(kps.size());
        IFGF_CUDA(cudaMemcpyAsync(D.kp_plane.p, kps.data(), kps.size() * sizeof(KParams),
                                  cudaMemcpyHostToDevice, st));
        IFGF_CUDA(cudaStreamSynchronize(st)); // kps is a temporary
        D.kp_host = kps;
    }
    BatchPtrs bp = batch_ptrs(in_plane, out_plane);
    bp.dgeo32 = D.dgeo32_ptr.data();
    set_batch_far(bp);
    MultPtrs m;
    fill_mult_ptrs(m);
    int64_t done = 0;
    while (done < nk)
    {
        bp.nrhs = (int)std::min<int64_t>(planes, nk - done);
        bp.groups = (bp.nrhs + BATCH_NB - 1) / BATCH_NB;
        bp.kp_plane = D.kp_plane.p + done;
        EventHooks log(D, st);
        int r = -1;
        IFGF_DISPATCH(kind_, r = launch_mult_batch_kernels<KK>(
                                 m, bp, (const double*)d_w + done * in_plane,
                                 (double*)d_u + done * out_plane, is_real(), st,
                                 profiling_ ? &log : nullptr));
        if (r < 0)
            throw Error(ERR_INVALID, "multi-wavenumber batches need one of the batched order "
                                     "shapes (low orders (2,5,5), (3,6,6) or (4,7,7))");
        launches_per_mult_ = r;
        if (profiling_ && log.n > 0)
            finish_profile(log, bp.nrhs);
        done += bp.nrhs;
    }
}

void Operator::host_mult_loop(const void* w, void* u, int64_t batch, int vkind)
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
        launch_mult(D.io_w.p, D.io_u.p, nullptr, false, vkind);
        IFGF_CUDA(cudaMemcpy((double*)u + b * nu, D.io_u.p, nu * sizeof(double),
                             cudaMemcpyDeviceToHost));
    }
    IFGF_CUDA(cudaMemcpy(&missing_, D.err.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    check_device_status();
}

void Operator::mult_device_external_scratch(const void* d_w, void* d_u, void* stream,
                                            void* scratch, size_t scratch_bytes)
{
    if (!initialized_)
        throw Error(ERR_STATE, "mult called before init");
    if (!d_w || !d_u || !scratch)
        throw Error(ERR_INVALID, "null density, result or scratch buffer");
    // the scratch is the current device's; the operator's tables must be there too
    int cur = -1;
    IFGF_CUDA(cudaGetDevice(&cur));
    if (cur != device_)
        throw Error(ERR_STATE, "the current device (" + std::to_string(cur) +
                                   ") is not the device this operator was initialised on (" +
                                   std::to_string(device_) + ")");
    DeviceState& D = *dev_;
    auto up = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t bw = up(D.w.n * sizeof(double2)), bc = up(D.cvals.n * sizeof(double2)),
                 bf = up(D.fcoef.n * sizeof(double2)), bn = up(D.unear.n * sizeof(double2));
    const size_t need = bw + bc + bf + bn;
    if (need > scratch_bytes)
        throw Error(ERR_INVALID, "this operator needs " + std::to_string(need) +
                                     " bytes of matvec scratch; the fixed no-allocation scratch "
                                     "holds " + std::to_string(scratch_bytes) +
                                     " bytes (use ifgf_mult_device for larger problems)");
    unsigned char* base = static_cast<unsigned char*>(scratch);
    double2* w = reinterpret_cast<double2*>(base);
    double2* cv = reinterpret_cast<double2*>(base + bw);
    double2* fc = reinterpret_cast<double2*>(base + bw + bc);
    double2* un = reinterpret_cast<double2*>(base + bw + bc + bf);
    cudaStream_t st = (cudaStream_t)stream;
    // fine cones without an active coarse parent must read as zero; the
    // shared scratch still holds the previous call's coefficients
    IFGF_CUDA(cudaMemsetAsync(fc, 0, D.fcoef.n * sizeof(double2), st));
    // point the operator's scratch buffers at the caller's region for this
    // call only (sizes unchanged), restoring them on every exit path
    struct Redirect
    {
        DeviceState& D;
        double2 *w, *cv, *fc, *un;
        ~Redirect()
        {
            D.w.p = w;
            D.cvals.p = cv;
            D.fcoef.p = fc;
            D.unear.p = un;
        }
    } restore{D, D.w.p, D.cvals.p, D.fcoef.p, D.unear.p};
    D.w.p = w;
    D.cvals.p = cv;
    D.fcoef.p = fc;
    D.unear.p = un;
    MultPtrs m;
    fill_mult_ptrs(m); // no hooks: this path creates no events
    IFGF_DISPATCH(kind_, launch_mult_kernels<KK>(m, d_w, d_u, is_real(), st, nullptr));
}

void Operator::direct_eval(const void* w, const int64_t* tidx, int64_t nt, void* out, bool dk)
{
    const int ek = dk ? dk_kind() : kind_;
    if (ek < 0)
        throw Error(ERR_INVALID, "the k-derivative exists for the Helmholtz and combined-field "
                                 "kernels only");
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
    DevBuf<int> dpos;
    dpos.upload(pos);
    DevBuf<double2> dout;
    dout.alloc(nt);
    MultPtrs m;
    fill_mult_ptrs(m);
    IFGF_DISPATCH(ek, permute_only<KK>(m, D.io_w.p, is_real(), nullptr);
                  launch_direct_kernel<KK>(m, dpos.p, (int)nt, dout.p, nullptr));
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
    // work the target-leaf lists describe, from the device tables of an
    // initialised operator (the host tables of a plan-only one)
    int64_t tl_work[4] = {0, 0, 0, 0};
    uint64_t tl_sum = 0;
    if (initialized_)
        plan_.target_list_work(dev_->tl_far_off.download(), dev_->tl_far_src.download(),
                               dev_->tl_near_off.download(), dev_->tl_near_src.download(),
                               tl_work, &tl_sum);
    else
        plan_.target_list_work(tl_work, &tl_sum);
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
      << ",\"far_point_pairs\":" << tl_work[3]
      << ",\"target_leaf_far_evals\":" << tl_work[0]
      << ",\"target_leaf_far_point_pairs\":" << tl_work[1]
      << ",\"target_leaf_near_point_pairs\":" << tl_work[2]
      << ",\"target_leaf_lists_checksum\":" << tl_sum
      << ",\"leaf_factor_evals\":" << leaf_evals_ << ",\"upward_node_evals\":" << upward_evals_
      << ",\"coarse_cones_total\":" << n_coarse_total_ << ",\"fine_cones_total\":" << n_fine_total_
      << ",\"upward_geometry_bytes\":" << upgeo_bytes_ << ",\"upward_runs_max\":[";
    for (size_t l = 0; l < fe_pad_.size(); l++)
        o << (l ? "," : "") << fe_pad_[l];
    o << "],\"upward_levels\":[";
    for (size_t l = 0; l < up_stats_.size(); l++)
        o << (l ? "," : "") << "{\"cones\":" << up_stats_[l].cones << ",\"slots\":"
          << up_stats_[l].slots << ",\"blocks\":" << up_stats_[l].blocks
          << ",\"padded_entries\":" << up_stats_[l].entries << "}";
    o << "]"
      << ",\"target_leaves\":" << dev_->n_tleaf << ",\"missing_cone_lookups\":" << missing_
      << ",\"init_ms\":" << init_ms_ << ",\"init_tree_ms\":" << tree_ms_
      << ",\"init_lists_ms\":" << lists_ms_ << ",\"init_target_lists_ms\":" << tlists_ms_
      << ",\"init_device_ms\":" << device_ms_ << ",\"init_device_phases_ms\":{";
    for (size_t i = 0; i < dev_phases_.size(); i++)
        o << (i ? "," : "") << "\"" << dev_phases_[i].first << "\":" << dev_phases_[i].second;
    o << "},\"far_plan\":{\"on\":" << (far_plan_on_ ? 1 : 0) << ",\"built\":"
      << (dev_->fp_ready ? 1 : 0) << ",\"chunks\":" << dev_->fp_nchunk
      << ",\"groups\":" << dev_->fp_group.n << ",\"records\":" << dev_->fp_rec.n
      << ",\"slot_entries\":" << dev_->fp_slot.n << ",\"bytes\":"
      << (dev_->fp_group.n * sizeof(FarGroup) + dev_->fp_rec.n * sizeof(FarPlanRec) +
          dev_->fp_slot.n * sizeof(int) + dev_->fp_chunk.n * sizeof(FarChunk))
      << ",\"slots_per_group\":" << dev_->fp_nslot << ",\"overflow_share_at_few_slots\":" << dev_->fp_ovf_few << ",\"build_ms\":" << dev_->fp_ms << "}";
    o << ",\"upward_images_bytes\":[";
    for (int l = 0; l < (int)lv_.size(); l++)
        o << (l ? "," : "") << (l < (int)dev_->tc_img.size() ? dev_->tc_img[l].n : 0);
    o << "]";
    o << ",\"upward_path\":" << up_path_ << ",\"upward_tuner\":{";
    {
        bool first = true;
        for (const auto& kv : dev_->up_choice)
        {
            auto arr = [&](const char* name, auto const& v) {
                o << "\"" << name << "\":[";
                for (size_t i = 0; i < v.size(); i++)
                    o << (i ? "," : "") << (double)v[i];
                o << "]";
            };
            o << (first ? "" : ",") << "\"" << kv.first << "\":{";
            arr("tensor", kv.second);
            o << ",";
            arr("ms_ffma", dev_->up_ms_ffma.at(kv.first));
            o << ",";
            arr("ms_tensor", dev_->up_ms_tc.at(kv.first));
            o << "}";
            first = false;
        }
    }
    o << "},\"launches_per_mult\":" << launches_per_mult_
      << ",\"batch_planes\":" << dev_->b_planes
      << ",\"last_mult_ms\":{\"permute\":" << last_.permute << ",\"leaf_sample\":" << last_.coarse
      << ",\"upward\":" << last_.upward << ",\"coarse_to_fine\":" << last_.c2f
      << ",\"target_eval\":" << last_.eval << ",\"near\":" << last_.near
      << ",\"total\":" << last_.total
      << "},\"profile\":{\"mults\":" << mults_profiled_;
    const char* names[NPROF] = {"permute", "leaf_sample", "coarse_to_fine", "target_eval",
                                "upward",  "near"};
    for (int i = 0; i < NPROF; i++)
    {
        o << ",\"" << names[i] << "\":{\"launches\":" << prof_launches_[i] << ",\"ms\":" << prof_ms_[i]
          << ",\"level_ms\":[";
        for (size_t l = 0; l < lv_.size(); l++)
            o << (l ? "," : "") << prof_level_ms_[i][l];
        o << "]}";
    }
    o << "}}";
    return o.str();
}

} // namespace ifgf
