// Upward transfer on the tensor cores (mixed precision, sm_100a tcgen05).
//
// The transfer of one level (transferInterp, ifgfoperator.hpp:1639-1705)
// evaluates, for every active coarse cone of a parent box and every child,
// the child's fine Chebyshev interpolant (P_LO = N0 N1 N2 complex
// coefficients) at the cone's high-order nodes, times the centre-shift
// factor, and sums over the children.  All boxes of a level have the same
// shape, so the node positions relative to a child -- its fine element, the
// local coordinates and the factor -- depend only on the parent element (the
// slot), the octant and the node (the level's geometry table).  Within one
// (slot, octant) row the nodes are sorted by child element into runs; every
// parent cone of the slot evaluates run r against ITS child's coefficient
// block of that element.  So for the cones of a slot, run r is a product
//
//     values[cone][entry] = sum_k coef[child(cone), element_r][k] * T_k(entry),
//
// with T_k(entry) = T_a(x) T_b(y) T_c(z) the tensor Chebyshev basis at the
// entry's local coordinates -- the same basis rows for every cone.  That is
// a GEMM with the cones (times right-hand-side planes) as M, the run's
// entries as N and the coefficients as K.
//
// One CTA takes a tile of 32 rows (cone, plane) of one slot.  The four
// lanes of a row in the 128-lane MMA are (real / imaginary part of the
// coefficients) x (TF32 high / low part of them) -- row 8 q + i of quarter q
// at lanes 32 q + 16 s + 8 p + i (part p, piece s), so that the 16-lane x
// 256-bit tensor-memory accesses hand one thread both parts of a row, and
// two of them both pieces, without shuffles.  A lives in tensor memory
// (K columns per lane), the basis in shared memory as 2 N rows -- the TF32
// high parts B_hi of the chunk's N entries, then their low parts B_lo -- so
// that one MMA per K step gives
//     D[lane][e] = A[lane] . B_hi[e],  D[lane][N + e] = A[lane] . B_lo[e]
// and summing both columns and the hi / lo lanes gives (A_hi + A_lo)(B_hi +
// B_lo), an FP32-accurate product (the 3xTF32 idea, with the splits carried
// by lanes and columns instead of extra MMAs).  D accumulates in FP32 in
// tensor memory.
//
// Warp roles (14 warps):
//   0-3   A producers: load a run's coefficient blocks (global memory, made
//         L2-resident by the loader) into tensor memory, split into TF32
//         high / low pieces
//   4-7   epilogue: read D, sum the hi / lo lanes, form the complex value,
//         multiply by the centre-shift factor and add it into the cone's
//         node accumulators (shared memory, FP32)
//   8-11  B producers: the basis rows of a chunk of <= 48 entries; with the
//         level's basis images (upward_tc_image_fill) one elected thread of
//         warp 8 copies the chunk's rows and entry data instead (two bulk
//         copies completing the same barriers by byte count)
//   12    loader: per run, the child fine cone of every row (looked up up
//         to four runs ahead) and an L2 prefetch of its coefficient block
//   13    lane 0 issues the MMAs (tcgen05.mma kind::tf32) and commits
// Pipelines: look-ups in four stages, A in two (per run), B and D in two
// (per chunk), all synchronised by mbarriers.  Every wait is
// bounded (global timer); a wait that gives up sets bit 0 of *tc_status and
// the CTA leaves its loops (the host reports IFGF_ERR_TIMEOUT).
//
// A tabulated element may be inactive in a child (the table works in
// coordinates relative to the parent, the cone activation in absolute ones,
// which can differ within one rounding of an element boundary); that row's
// A lanes are zero and the epilogue evaluates its entries from absolute
// coordinates on the CUDA cores, as the FFMA kernels do.
#pragma once

#include "tcgen05.cuh"

namespace ifgf
{

constexpr int UPTC_ROWS = 32;     // rows (cone, plane) per tile
constexpr int UPTC_NMAX = 48;     // entries per chunk (MMA N <= 48)
constexpr int UPTC_THREADS = 448; // 14 warps
constexpr unsigned long long UPTC_WAIT_NS = 2000000000ull; // 2 s per wait
// tensor-memory columns: A stages at 0 / 128, D stages (2 x 48 columns:
// high- and low-part basis) at 256 / 352
constexpr int UPTC_TM_A = 0, UPTC_TM_A_STRIDE = 128, UPTC_TM_D = 256, UPTC_TM_D_STRIDE = 96;
constexpr int UPTC_TM_COLS = 512;
// shared memory below which two CTAs could share an SM (and then wait for
// each other's tensor-memory columns): every launch asks for at least this
constexpr size_t UPTC_SMEM_MIN = 120 * 1024;

// mbarrier indices
enum UpTcBar
{
    UTB_ROW_FULL = 0,   // [4] a run's fine cones looked up (loader)
    UTB_ROW_EMPTY = 4,  // [4] A producers done with them (4 arrivals)
    UTB_A_FULL = 8,     // [2] A stage written to tensor memory (4 arrivals)
    UTB_A_EMPTY = 10,   // [2] MMAs of the run done (commit)
    UTB_B_FULL = 12,    // [2] B stage written (4 arrivals)
    UTB_B_EMPTY = 14,   // [2] MMAs of the chunk done (commit)
    UTB_D_FULL = 16,    // [2] D stage complete (commit)
    UTB_D_EMPTY = 18,   // [2] epilogue done with the D stage and its entry data (4 arrivals)
    UTB_META_FULL = 20, // [2] a chunk's entry data (node, factor) written (4 arrivals)
    UTB_COUNT = 22
};
constexpr int UPTC_ROW_STAGES = 4; // look-up stages the loader runs ahead of the A producers

// Row flags of a run: which rows have a staged coefficient block.
constexpr int UPTC_NONE = -1;     // no child at this octant, or a padding row
constexpr int UPTC_FALLBACK = -2; // element inactive in the child: CUDA-core path
constexpr int UPTC_END = -3;      // loader look-up slot past the tile's last run

struct UpTcLayout
{
    size_t b, acc, meta, rowgf, rowinfo, runs, bars, total;
    int rs; // accumulator row stride (floats, odd)
};

template <int N0, int N1, int N2> struct UpTcShape
{
    static constexpr int P_LO = N0 * N1 * N2;
    static constexpr int K = (P_LO + 7) / 8 * 8; // MMA K steps of 8
    static constexpr int KS = K / 8;
    static constexpr int RAW_ROW = P_LO * 8;       // bytes of one coefficient block (L2 prefetch)
    static constexpr int B_BYTES = 2 * UPTC_NMAX * K * 4; // B_hi and B_lo rows of a chunk
    static constexpr int SBO = (K / 4) * 128;      // bytes between 8-row groups of B
    static_assert(K <= UPTC_TM_A_STRIDE, "coefficient blocks wider than a tensor-memory stage");
    static_assert(RAW_ROW % 16 == 0, "bulk prefetches move multiples of 16 bytes");
    static_assert(UPTC_NMAX % 16 == 0 && 2 * UPTC_NMAX <= UPTC_TM_D_STRIDE, "chunk width");
};

template <int N0, int N1, int N2>
inline __host__ __device__ UpTcLayout uptc_layout(int P_hi, int fe_pad)
{
    using S = UpTcShape<N0, N1, N2>;
    auto al = [](size_t x) { return (x + 15) / 16 * 16; };
    UpTcLayout L{};
    L.rs = P_hi | 1;
    size_t o = 0;
    L.b = o; // two stages
    o = al(o + 2 * (size_t)S::B_BYTES);
    L.acc = o;
    o = al(o + 2 * ((size_t)UPTC_ROWS * L.rs + 16) * sizeof(float));
    L.meta = o; // [2][NMAX] (node, factor re, factor im, -)
    o = al(o + 2 * (size_t)UPTC_NMAX * 16);
    L.rowgf = o; // [UPTC_ROW_STAGES][ROWS]
    o = al(o + UPTC_ROW_STAGES * (size_t)UPTC_ROWS * 4);
    L.rowinfo = o; // cone, plane, box, child[8] per row; octant used [8]
    o = al(o + (size_t)UPTC_ROWS * 11 * 4 + 8 * 4);
    L.runs = o; // [8][fe_pad + 1] int2, then row_n[16]
    o = al(o + (size_t)8 * (fe_pad + 1) * 8 + 16 * 4);
    L.bars = o; // the mbarriers, then the tensor-memory base address
    o = al(o + UTB_COUNT * 8 + 16);
    L.total = o;
    return L;
}

// Dynamic shared memory of a launch (at least UPTC_SMEM_MIN, so that one CTA
// holds an SM and its tensor-memory allocation never waits).
template <int N0, int N1, int N2> inline size_t uptc_smem_bytes(int P_hi, int fe_pad)
{
    const size_t total = uptc_layout<N0, N1, N2>(P_hi, fe_pad).total;
    return total < UPTC_SMEM_MIN ? UPTC_SMEM_MIN : total;
}

// Basis row of one entry for the K columns [H * K / 2, (H + 1) * K / 2):
// TF32 high parts into bh, low parts into bl (the K-major core-matrix layout
// of the B operand; column group k / 4 at 32-float steps).  Compile-time H
// keeps every index a constant.
template <int N0, int N1, int N2, int H>
__device__ __forceinline__ void uptc_basis_half(bool live, float x0, float x1, float x2,
                                                float* bh, float* bl)
{
    constexpr int P_LO = N0 * N1 * N2;
    constexpr int KH = UpTcShape<N0, N1, N2>::K / 2;
    float t0[N0], t1[N1], t2[N2];
    cheb_basis<float, N0>(x0, t0);
    cheb_basis<float, N1>(x1, t1);
    cheb_basis<float, N2>(x2, t2);
#pragma unroll
    for (int k4 = 0; k4 < KH; k4 += 4)
    {
        float hv[4], lv[4];
#pragma unroll
        for (int j = 0; j < 4; j++)
        {
            const int k = H * KH + k4 + j;
            float v = 0.f;
            if (k < P_LO)
                v = live ? t0[k % N0] * t1[(k / N0) % N1] * t2[k / (N0 * N1)] : 0.f;
            hv[j] = tc::tf32_round(v);
            lv[j] = v - hv[j];
        }
        const int kk = H * KH + k4;
        *reinterpret_cast<float4*>(bh + (kk >> 2) * 32) = make_float4(hv[0], hv[1], hv[2], hv[3]);
        *reinterpret_cast<float4*>(bl + (kk >> 2) * 32) = make_float4(lv[0], lv[1], lv[2], lv[3]);
    }
}

// The upward contribution of one table entry (parent node `node` of cone
// element `el` of box `box`, child `cb`) evaluated from absolute coordinates
// on the CUDA cores, as the FFMA kernels do: for a tabulated element that is
// inactive in the child.  Out of line: it runs rarely and its code would
// otherwise crowd the instruction cache of the pipelined roles.
template <int KIND, int N0, int N1, int N2>
__device__ __noinline__ cplx<float> uptc_fallback(const UpArgs& a, int box, int el, int node,
                                                  int cb, const float2* fcq)
{
    const LevelGeom& C = a.GC;
    const long long nf = (long long)C.nf[0] * C.nf[1] * C.nf[2];
    const double xc[3] = {a.T.box_c[3 * box], a.T.box_c[3 * box + 1], a.T.box_c[3 * box + 2]};
    double y[3];
    node_position(a.G, el, node, a.hi_nodes, xc, a.T.box_H[box], y);
    const double p[3] = {y[0] - a.T.box_c[3 * cb], y[1] - a.T.box_c[3 * cb + 1],
                         y[2] - a.T.box_c[3 * cb + 2]};
    float loc[3];
    const int* fm = a.fmap + C.fmap_off + (long long)(cb - C.box_off) * nf;
    const int gf2 = fine_lookup_mixed(C, fm, p, a.T.box_H[cb], loc, a.err);
    cplx<float> val = {0.f, 0.f};
    if (gf2 < 0)
        return val;
    const double e0 = y[0] - xc[0], e1 = y[1] - xc[1], e2 = y[2] - xc[2];
    cfmaf(val, ChebF<N0, N1, N2>::eval(fcq + (size_t)gf2 * (N0 * N1 * N2), loc, a.lo),
          transfer_mixed<KIND>(p[0] * p[0] + p[1] * p[1] + p[2] * p[2],
                               e0 * e0 + e1 * e1 + e2 * e2, a.kp));
    return val;
}

template <int KIND, int N0, int N1, int N2>
__global__ void __launch_bounds__(UPTC_THREADS, 1) upward_tc_kernel(const __grid_constant__ UpArgs a)
{
    using S = UpTcShape<N0, N1, N2>;
    constexpr int P_LO = S::P_LO, K = S::K, KS = S::KS;
    constexpr int GMAX = UPTC_NMAX / UPGEO_RUN; // groups per chunk
    extern __shared__ __align__(1024) unsigned char uptc_sm[];
    unsigned char* sm = uptc_sm;
    const UpTcLayout LY = uptc_layout<N0, N1, N2>(a.P_hi, a.fe_pad);
    float* Bs = reinterpret_cast<float*>(sm + LY.b);
    float* acc = reinterpret_cast<float*>(sm + LY.acc);
    int4* meta = reinterpret_cast<int4*>(sm + LY.meta);
    int* rowgf = reinterpret_cast<int*>(sm + LY.rowgf);
    int* row_c = reinterpret_cast<int*>(sm + LY.rowinfo);
    int* row_q = row_c + UPTC_ROWS;
    int* row_box = row_q + UPTC_ROWS;
    int* row_cb = row_box + UPTC_ROWS; // [ROWS][8]
    int* used = row_cb + 8 * UPTC_ROWS;
    int2* fl = reinterpret_cast<int2*>(sm + LY.runs);
    const int FL = a.fe_pad + 1;
    int* row_n = reinterpret_cast<int*>(fl + 8 * FL);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(sm + LY.bars);
    unsigned* tbase_sm = reinterpret_cast<unsigned*>(bars + UTB_COUNT);
    const int RS = LY.rs;
    const int accp = UPTC_ROWS * RS + 16; // floats between the real and imaginary accumulators

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int4 tile = a.tc_tiles[blockIdx.x]; // (first up_idx position, cones, first plane, planes)
    const int nrows = tile.y * tile.w;
    const int ngroups = a.P_pad / UPGEO_RUN;
    const LevelGeom& C = a.GC;
    const long long nf = (long long)C.nf[0] * C.nf[1] * C.nf[2];
    const float2* fc2 = reinterpret_cast<const float2*>(a.fcoef);
    const int slot = a.slot[tile.x];
    const int el = a.cc_el[a.idx[tile.x]];

    // ---- set-up: row tables, run lists, accumulators, barriers, TMEM ----
    if (tid < UPTC_ROWS)
    {
        const int i = tid;
        if (i < nrows)
        {
            const int c = a.idx[tile.x + i / tile.w];
            const int box = a.cc_box[c];
            row_c[i] = c;
            row_q[i] = tile.z + i % tile.w;
            row_box[i] = box;
            for (int o = 0; o < 8; o++)
                row_cb[8 * i + o] = a.T.box_child[8 * box + o];
        }
        else
        {
            row_c[i] = -1;
            row_q[i] = 0;
            row_box[i] = -1;
            for (int o = 0; o < 8; o++)
                row_cb[8 * i + o] = -1;
        }
    }
    if (tid >= 64 && tid < 72)
    {
        row_n[tid - 64] = a.fe_pad;
        row_n[8 + tid - 64] = ngroups;
    }
    for (int i = tid; i < 2 * accp; i += blockDim.x)
        acc[i] = 0.f;
    if (tid == 96)
    {
        for (int b = 0; b < UTB_COUNT; b++)
        {
            unsigned cnt = 1;
            if ((b >= UTB_ROW_EMPTY && b < UTB_ROW_EMPTY + UPTC_ROW_STAGES) ||
                b == UTB_A_FULL || b == UTB_A_FULL + 1 || b == UTB_D_EMPTY || b == UTB_D_EMPTY + 1)
                cnt = 4;
            if (b == UTB_B_FULL || b == UTB_B_FULL + 1 || b == UTB_META_FULL ||
                b == UTB_META_FULL + 1)
                cnt = a.tc_img ? 1 : 4; // one bulk-copy issuer, or four producer warps
            tc::mbar_init(tc::smem_u32(bars + b), cnt);
        }
        tc::mbar_init_fence();
    }
    if (warp == 13)
        tc::tmem_alloc(tc::smem_u32(tbase_sm), UPTC_TM_COLS);
    __syncthreads();
    for (int i = tid; i < 8 * FL; i += blockDim.x)
    {
        const int o = i / FL, r = i - o * FL;
        const int2 f = a.fe_list[((size_t)slot * 8 + o) * FL + r];
        fl[i] = f;
        if (f.x < 0 && f.y >= 0)
        {
            // the sentinel after the row's last run: (-1, groups of the row)
            row_n[o] = r;
            row_n[8 + o] = f.y;
        }
    }
    if (tid < 8)
    {
        int u = 0;
        for (int i = 0; i < nrows; i++)
            u |= row_cb[8 * i + tid] >= 0;
        used[tid] = u;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const unsigned tbase = *tbase_sm;
    auto bar = [&](int b) { return tc::smem_u32(bars + b); };
    bool ok = true;

    // (octant, run) -> element, first and end group
    auto run_info = [&](int o, int r, int& ce, int& g0, int& g1) {
        const int2 f = fl[o * FL + r];
        ce = f.x;
        g0 = f.y;
        g1 = r + 1 < row_n[o] ? fl[o * FL + r + 1].y : row_n[8 + o];
    };
    // child fine cone of row i for octant o, element ce
    auto row_block = [&](int i, int o, int ce) -> int {
        const int cb = row_cb[8 * i + o];
        if (cb < 0)
            return UPTC_NONE;
        const int gf = a.fmap[C.fmap_off + (long long)(cb - C.box_off) * nf + ce];
        return gf >= 0 ? gf : UPTC_FALLBACK;
    };

    if (warp == 12)
    {
        // ---------------- loader ----------------
        // The fine-cone lookups (a dependent, often uncached global load per
        // row) run four runs ahead of their use: the loop is unrolled four
        // times so that look-up slot i (a register) is read only by step i,
        // four runs after its load was issued.
        auto next_run = [&](int& qo, int& qr) -> bool {
            for (; qo < 8; qo++, qr = 0)
                if (used[qo] && qr < row_n[qo])
                    return true;
            return false;
        };
        int io = 0, ir = 0; // the next run to look up
        auto issue = [&](int& slot_gf) {
            slot_gf = UPTC_END;
            if (next_run(io, ir))
            {
                int ce, g0, g1;
                run_info(io, ir, ce, g0, g1);
                slot_gf = row_block(lane, io, ce);
                ir++;
            }
        };
        int lgf0, lgf1, lgf2, lgf3;
        issue(lgf0);
        issue(lgf1);
        issue(lgf2);
        issue(lgf3);
        int R = 0;
        auto step = [&](int& slot_gf) -> bool {
            const int gf = slot_gf;
            if (gf == UPTC_END)
                return false;
            issue(slot_gf);
            const int st = R % UPTC_ROW_STAGES, ph = R / UPTC_ROW_STAGES;
            if (R >= UPTC_ROW_STAGES &&
                !tc::mbar_wait(bar(UTB_ROW_EMPTY + st), (ph - 1) & 1, UPTC_WAIT_NS))
            {
                ok = false;
                return false;
            }
            if (gf >= 0)
                tc::prefetch_l2(fc2 + (size_t)row_q[lane] * a.fc_plane + (size_t)gf * P_LO,
                                (unsigned)S::RAW_ROW);
            rowgf[st * UPTC_ROWS + lane] = gf;
            __syncwarp();
            if (lane == 0)
                tc::mbar_arrive(bar(UTB_ROW_FULL + st));
            R++;
            return true;
        };
        while (step(lgf0) && step(lgf1) && step(lgf2) && step(lgf3))
        {
        }
        if (!ok && lane == 0)
            atomicOr(a.tc_status, 1u);
    }
    else if (warp < 4)
    {
        // ---------------- A producers ----------------
        // warp q writes rows 8 q .. 8 q + 7: thread t takes row 8 q + t / 4 and,
        // per group of 8 coefficients, the pair 2 (t % 4), 2 (t % 4) + 1 -- one
        // 16-byte load gives both parts of both, stored to the high-piece lanes
        // (16 s = 0) and the low-piece lanes (16 s = 16) of the row
        const int ri = 8 * warp + (lane >> 2), t0 = lane & 3;
        const unsigned lane_base = tbase + ((unsigned)(32 * warp) << 16);
        int R = 0;
        for (int o = 0; o < 8 && ok; o++)
        {
            if (!used[o])
                continue;
            for (int r = 0; r < row_n[o]; r++, R++)
            {
                const int st = R & 1;
                const int rs = R % UPTC_ROW_STAGES;
                if (!tc::mbar_wait(bar(UTB_ROW_FULL + rs), (R / UPTC_ROW_STAGES) & 1, UPTC_WAIT_NS) ||
                    (R >= 2 && !tc::mbar_wait(bar(UTB_A_EMPTY + st), ((R >> 1) - 1) & 1, UPTC_WAIT_NS)))
                {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const int gf = rowgf[rs * UPTC_ROWS + ri];
                __syncwarp();
                if (lane == 0)
                    tc::mbar_arrive(bar(UTB_ROW_EMPTY + rs));
                const float4* src4 = reinterpret_cast<const float4*>(
                    fc2 + (size_t)row_q[ri] * a.fc_plane + (size_t)(gf >= 0 ? gf : 0) * P_LO);
                const unsigned col = UPTC_TM_A + st * UPTC_TM_A_STRIDE;
                // all of this thread's coefficient pairs in flight at once
                float4 c4[K / 8];
#pragma unroll
                for (int g = 0; g < K / 8; g++)
                {
                    const int k = 8 * g + 2 * t0; // the coefficient pair of this thread
                    c4[g] = (gf >= 0 && k < P_LO) ? __ldg(src4 + (k >> 1))
                                                  : make_float4(0.f, 0.f, 0.f, 0.f);
                }
#pragma unroll
                for (int g = 0; g < K / 8; g++)
                {
                    const float h0 = tc::tf32_round(c4[g].x), h1 = tc::tf32_round(c4[g].z);
                    const float h2 = tc::tf32_round(c4[g].y), h3 = tc::tf32_round(c4[g].w);
                    // (real k, real k + 1) -> lane of part 0, (imag k, imag k + 1) -> part 1
                    tc::tmem_st16x256(lane_base + col + 8 * g, __float_as_uint(h0),
                                      __float_as_uint(h1), __float_as_uint(h2), __float_as_uint(h3));
                    tc::tmem_st16x256(lane_base + (16u << 16) + col + 8 * g,
                                      __float_as_uint(c4[g].x - h0), __float_as_uint(c4[g].z - h1),
                                      __float_as_uint(c4[g].y - h2), __float_as_uint(c4[g].w - h3));
                }
                tc::tmem_wait_st();
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0)
                    tc::mbar_arrive(bar(UTB_A_FULL + st));
            }
        }
        if (!ok && lane == 0)
            atomicOr(a.tc_status, 1u);
    }
    else if (warp >= 8 && warp < 12 && a.tc_img)
    {
        // ---------------- B operand and entry data from the basis images ----------------
        // the walk of the MMA issuer; per chunk, once its stage is free, one
        // lane copies the record (entry data, then the B rows) of the image
        if (warp == 8)
        {
            int Cn = 0;
            for (int o = 0; o < 8 && ok; o++)
            {
                if (!used[o])
                    continue;
                long long pos = a.tc_img_off[(size_t)slot * 8 + o];
                for (int r = 0; r < row_n[o] && ok; r++)
                {
                    int ce, g0, g1;
                    run_info(o, r, ce, g0, g1);
                    for (int cg = g0; cg < g1; cg += GMAX, Cn++)
                    {
                        const int nent = UPGEO_RUN * min(GMAX, g1 - cg);
                        const int N = (nent + 15) & ~15;
                        const int bs = Cn & 1;
                        if (Cn >= 2 &&
                            (!tc::mbar_wait(bar(UTB_B_EMPTY + bs), ((Cn >> 1) - 1) & 1,
                                            UPTC_WAIT_NS) ||
                             !tc::mbar_wait(bar(UTB_D_EMPTY + bs), ((Cn >> 1) - 1) & 1,
                                            UPTC_WAIT_NS)))
                        {
                            ok = false;
                            break;
                        }
                        if (tc::elect_one())
                        {
                            const unsigned mbytes = 16u * N, bbytes = 8u * N * K;
                            tc::mbar_arrive_expect_tx(bar(UTB_META_FULL + bs), mbytes);
                            tc::bulk_g2s(tc::smem_u32(meta + bs * UPTC_NMAX), a.tc_img + pos, mbytes,
                                         bar(UTB_META_FULL + bs));
                            tc::mbar_arrive_expect_tx(bar(UTB_B_FULL + bs), bbytes);
                            tc::bulk_g2s(tc::smem_u32(Bs + (size_t)bs * (S::B_BYTES / 4)),
                                         a.tc_img + pos + mbytes, bbytes, bar(UTB_B_FULL + bs));
                        }
                        __syncwarp();
                        pos += (long long)N * (16 + 8 * K);
                    }
                }
            }
            if (!ok && lane == 0)
                atomicOr(a.tc_status, 1u);
        }
    }
    else if (warp >= 8 && warp < 12)
    {
        // ---------------- B producers ----------------
        const int tb = tid - 256;              // 0..127
        const int half = tb >> 6, e = tb & 63; // K half, entry of the chunk
        // the (octant, run, chunk) walk, one chunk ahead: the next chunk's
        // table entry is loaded before this chunk's buffer is free
        int o = 0, r = 0, cg = 0, g1 = 0, ce = 0, g0 = 0;
        auto next_chunk = [&](int& po, int& pr, int& pcg, int& pg1) -> bool {
            // advance (po, pr, pcg) to the next chunk; false at the end
            if (pcg >= 0)
            {
                pcg += GMAX;
                if (pcg < pg1)
                    return true;
                pr++;
            }
            for (; po < 8; po++, pr = 0)
            {
                if (!used[po] || pr >= row_n[po])
                    continue;
                run_info(po, pr, ce, g0, pg1);
                pcg = g0;
                return true;
            }
            return false;
        };
        cg = -1;
        bool have = next_chunk(o, r, cg, g1);
        UpGeo32 gnext;
        auto load_entry = [&](int po, int pcg, int pg1, UpGeo32& g) {
            const int nent = UPGEO_RUN * min(GMAX, pg1 - pcg);
            g.node = -1;
            if (e < nent)
                g = a.geo32[((size_t)slot * 8 + po) * a.P_pad + (size_t)(e % UPGEO_RUN) * ngroups +
                            pcg + e / UPGEO_RUN];
        };
        if (have)
            load_entry(o, cg, g1, gnext);
        for (int Cn = 0; have && ok; Cn++)
        {
            const UpGeo32 g = gnext;
            const int co = o, ccg = cg, cg1 = g1;
            have = next_chunk(o, r, cg, g1);
            if (have)
                load_entry(o, cg, g1, gnext);
            const int nent = UPGEO_RUN * min(GMAX, cg1 - ccg);
            const int N = (nent + 15) & ~15;
            (void)co;
            const int bs = Cn & 1; // B stage; also the stage of the entry data
            if (Cn >= 2 &&
                (!tc::mbar_wait(bar(UTB_B_EMPTY + bs), ((Cn >> 1) - 1) & 1, UPTC_WAIT_NS) ||
                 !tc::mbar_wait(bar(UTB_D_EMPTY + bs), ((Cn >> 1) - 1) & 1, UPTC_WAIT_NS)))
            {
                ok = false;
                break;
            }
            float* Bst = Bs + (size_t)bs * (S::B_BYTES / 4);
            if (e < N)
            {
                const int node = e < nent ? g.node : -1;
                // high part at row e, low part at row N + e
                float* bh = Bst + (size_t)(e >> 3) * (S::SBO / 4) + (e & 7) * 4;
                float* bl = Bst + (size_t)((N + e) >> 3) * (S::SBO / 4) + ((N + e) & 7) * 4;
                if (half == 0)
                    uptc_basis_half<N0, N1, N2, 0>(node >= 0, g.loc[0], g.loc[1], g.loc[2], bh, bl);
                else
                    uptc_basis_half<N0, N1, N2, 1>(node >= 0, g.loc[0], g.loc[1], g.loc[2], bh, bl);
                if (half == 0)
                    meta[(Cn & 1) * UPTC_NMAX + e] =
                        make_int4(node, __float_as_int(g.tr), __float_as_int(g.ti), 0);
            }
            tc::fence_proxy_async();
            __syncwarp();
            if (lane == 0)
            {
                tc::mbar_arrive(bar(UTB_B_FULL + bs));
                tc::mbar_arrive(bar(UTB_META_FULL + bs));
            }
        }
        if (!ok && lane == 0)
            atomicOr(a.tc_status, 1u);
    }
    else if (warp == 13)
    {
        // ---------------- MMA issuer ----------------
        // The whole warp walks the sequence and waits (converged); one
        // elected lane issues each chunk's fully unrolled K loop.  Issued
        // from a diverged single thread, every MMA took ~3x as long.
        int R = 0, Cn = 0;
        unsigned last_bar = 0, last_par = 0;
        bool issued = false;
        const unsigned bb = tc::smem_u32(Bs);
        for (int o = 0; o < 8 && ok; o++)
        {
            if (!used[o])
                continue;
            for (int r = 0; r < row_n[o] && ok; r++, R++)
            {
                int ce, g0, g1;
                run_info(o, r, ce, g0, g1);
                const int st = R & 1;
                if (!tc::mbar_wait(bar(UTB_A_FULL + st), (R >> 1) & 1, UPTC_WAIT_NS))
                {
                    ok = false;
                    break;
                }
                for (int cg = g0; cg < g1; cg += GMAX, Cn++)
                {
                    const int nent = UPGEO_RUN * min(GMAX, g1 - cg);
                    const int N = (nent + 15) & ~15;
                    const int ds = Cn & 1;
                    if (!tc::mbar_wait(bar(UTB_B_FULL + ds), (Cn >> 1) & 1, UPTC_WAIT_NS) ||
                        (Cn >= 2 &&
                         !tc::mbar_wait(bar(UTB_D_EMPTY + ds), ((Cn >> 1) - 1) & 1, UPTC_WAIT_NS)))
                    {
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                    // rows [0, N): B_hi, [N, 2N): B_lo of the chunk's entries
                    const unsigned idesc = tc::idesc_tf32(128, 2 * N);
                    const unsigned dcol = tbase + UPTC_TM_D + ds * UPTC_TM_D_STRIDE;
                    const unsigned acol = tbase + UPTC_TM_A + st * UPTC_TM_A_STRIDE;
                    const bool last = cg + GMAX >= g1;
                    if (tc::elect_one())
                    {
#pragma unroll
                        for (int s = 0; s < KS; s++)
                            tc::mma_tf32_ts(dcol, acol + 8 * s,
                                            tc::smem_desc(bb + ds * S::B_BYTES + 256 * s, 128, S::SBO),
                                            idesc, s != 0);
                        tc::mma_commit(bar(UTB_B_EMPTY + ds));
                        tc::mma_commit(bar(UTB_D_FULL + ds));
                        if (last)
                            tc::mma_commit(bar(UTB_A_EMPTY + st));
                    }
                    __syncwarp();
                    last_bar = bar(UTB_D_FULL + ds);
                    last_par = (Cn >> 1) & 1;
                    issued = true;
                }
            }
        }
        if (!ok)
        {
            if (lane == 0)
                atomicOr(a.tc_status, 1u);
            // leave no MMA in flight
            if (issued)
                tc::mbar_wait(last_bar, last_par, UPTC_WAIT_NS);
        }
    }
    else
    {
        // ---------------- epilogue (warps 4-7) ----------------
        // warp 4 + q reads rows 8 q .. 8 q + 7: thread t takes row 8 q + t / 4
        // and, per group of 8 entries, entries 2 (t % 4) and 2 (t % 4) + 1, for
        // which four 16x256b loads (TF32 piece s of A x high / low rows of B)
        // give both parts; their sum is the full value, with no shuffles
        const int q = warp - 4;
        const int ri = 8 * q + (lane >> 2), t0 = lane & 3;
        const bool valid = ri < nrows;
        float* acc_re = acc + ri * RS;
        float* acc_im = acc_re + accp;
        const float2* fcq = fc2 + (size_t)row_q[ri] * a.fc_plane;
        const unsigned lane_base = tbase + ((unsigned)(32 * q) << 16);
        int Cn = 0;
        // row flag of the next run, looked up one run ahead
        int po = 0, pr = 0, pce = 0, pg0 = 0, pg1 = 0;
        auto next_run = [&](int& qo, int& qr) -> bool {
            for (; qo < 8; qo++, qr = 0)
                if (used[qo] && qr < row_n[qo])
                    return true;
            return false;
        };
        bool more = next_run(po, pr);
        int flag_next = UPTC_NONE;
        if (more)
        {
            run_info(po, pr, pce, pg0, pg1);
            flag_next = valid ? row_block(ri, po, pce) : UPTC_NONE;
        }
        while (more && ok)
        {
            const int o = po, g0 = pg0, g1 = pg1, flag = flag_next;
            pr++;
            more = next_run(po, pr);
            if (more)
            {
                run_info(po, pr, pce, pg0, pg1);
                flag_next = valid ? row_block(ri, po, pce) : UPTC_NONE;
            }
            const int cb = row_cb[8 * ri + o];
            for (int cg = g0; cg < g1; cg += GMAX, Cn++)
            {
                const int nent = UPGEO_RUN * min(GMAX, g1 - cg);
                const int N = (nent + 15) & ~15;
                const int ds = Cn & 1;
                // the entry data comes straight from the B producers (its own
                // barrier); D from the MMA completion
                if (!tc::mbar_wait(bar(UTB_META_FULL + ds), (Cn >> 1) & 1, UPTC_WAIT_NS) ||
                    !tc::mbar_wait(bar(UTB_D_FULL + ds), (Cn >> 1) & 1, UPTC_WAIT_NS))
                {
                    ok = false;
                    break;
                }
                tc::fence_after_sync();
                const int4* mt = meta + ds * UPTC_NMAX;
                const unsigned dcol = UPTC_TM_D + ds * UPTC_TM_D_STRIDE;
                // 16 entries at a time (two groups of 8; the chunk is padded to a
                // multiple of 16 columns, so both groups' loads are in range):
                // eight tensor-memory loads, one wait; then this thread's four
                // entries -- distinct nodes, so all accumulator loads are issued
                // before any store
                auto load_group = [&](int g, unsigned (&x)[4][4]) {
                    tc::tmem_ld16x256(lane_base + dcol + g, x[0]);                  // A_hi . B_hi
                    tc::tmem_ld16x256(lane_base + dcol + N + g, x[1]);              // A_hi . B_lo
                    tc::tmem_ld16x256(lane_base + (16u << 16) + dcol + g, x[2]);     // A_lo . B_hi
                    tc::tmem_ld16x256(lane_base + (16u << 16) + dcol + N + g, x[3]); // A_lo . B_lo
                };
#pragma unroll 1
                for (int g = 0; g < nent; g += 16)
                {
                    unsigned u[2][4][4];
                    load_group(g, u[0]);
                    load_group(g + 8, u[1]);
                    int nd[4];
                    float fr[4], fi[4];
#pragma unroll
                    for (int j = 0; j < 4; j++)
                    {
                        // entries g + 2 t0 + {0, 1} and g + 8 + 2 t0 + {0, 1}
                        const int e = g + 8 * (j >> 1) + 2 * t0 + (j & 1);
                        const int4 m = mt[min(e, UPTC_NMAX - 1)];
                        nd[j] = (flag >= 0 && e < nent) ? m.x : -1;
                        fr[j] = __int_as_float(m.y);
                        fi[j] = __int_as_float(m.z);
                    }
                    float ar[4], ai[4];
#pragma unroll
                    for (int j = 0; j < 4; j++)
                    {
                        ar[j] = nd[j] >= 0 ? acc_re[nd[j]] : 0.f;
                        ai[j] = nd[j] >= 0 ? acc_im[nd[j]] : 0.f;
                    }
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int j = 0; j < 4; j++)
                    {
                        const unsigned(&x)[4][4] = u[j >> 1];
                        const int h = j & 1;
                        // (re, im) of the entry: the four TF32 products summed
                        const float re = (__uint_as_float(x[0][h]) + __uint_as_float(x[1][h])) +
                                         (__uint_as_float(x[2][h]) + __uint_as_float(x[3][h]));
                        const float im =
                            (__uint_as_float(x[0][2 + h]) + __uint_as_float(x[1][2 + h])) +
                            (__uint_as_float(x[2][2 + h]) + __uint_as_float(x[3][2 + h]));
                        if (nd[j] >= 0)
                        {
                            acc_re[nd[j]] = ar[j] + (re * fr[j] - im * fi[j]);
                            acc_im[nd[j]] = ai[j] + (re * fi[j] + im * fr[j]);
                        }
                    }
                }
                if (flag == UPTC_FALLBACK)
                    for (int e = t0; e < nent; e += 4)
                    {
                        const int node = mt[e].x;
                        if (node < 0)
                            continue;
                        const cplx<float> val =
                            uptc_fallback<KIND, N0, N1, N2>(a, row_box[ri], el, node, cb, fcq);
                        acc_re[node] += val.re;
                        acc_im[node] += val.im;
                    }
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0)
                    tc::mbar_arrive(bar(UTB_D_EMPTY + ds));
            }
        }
        if (!ok && lane == 0)
            atomicOr(a.tc_status, 1u);
    }

    // ---- write the accumulated node values (plane q, cone c) ----
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    float2* cv = reinterpret_cast<float2*>(a.cvals);
    for (int i = 0; i < nrows; i++)
    {
        float2* out = cv + (size_t)row_q[i] * a.cv_plane + (size_t)row_c[i] * a.P_hi;
        const float* ar = acc + i * RS;
        for (int n = tid; n < a.P_hi; n += blockDim.x)
            out[n] = make_float2(ar[n], ar[accp + n]);
    }
    if (warp == 13)
        tc::tmem_dealloc(tbase, UPTC_TM_COLS);
}

// Basis images of one level (upward_tc_image_sizes / _fill, mult.hpp): one
// CTA per (slot, octant) row, walking its runs and chunks as the kernel does;
// per chunk of nent entries (N = nent rounded up to 16) the record is the
// entry data (N x int4: node, centre-shift factor) followed by the B stage
// image (2 N x K floats: TF32 high parts of the basis rows, then low parts,
// in the K-major core-matrix layout), exactly what the B producers would
// write to shared memory.  sizes != null: only the row's bytes.  meta_only:
// only the entry data (the centre-shift factors follow the wavenumber, the
// basis rows do not).
template <int N0, int N1, int N2>
__global__ void __launch_bounds__(128)
    uptc_image_kernel(const int2* __restrict__ fe_list, int fe_pad,
                      const UpGeo32* __restrict__ geo32, int P_pad,
                      const long long* __restrict__ off, unsigned char* img, long long* sizes,
                      bool meta_only)
{
    using S = UpTcShape<N0, N1, N2>;
    constexpr int K = S::K;
    constexpr int GMAX = UPTC_NMAX / UPGEO_RUN;
    const int so = blockIdx.x, o = so & 7;
    const size_t slot = (size_t)(so >> 3);
    const int FL = fe_pad + 1, ngroups = P_pad / UPGEO_RUN;
    const int2* fl = fe_list + (size_t)so * FL;
    int nrun = fe_pad, rgroups = ngroups;
    for (int r = 0; r < FL; r++)
    {
        const int2 f = fl[r];
        if (f.x < 0 && f.y >= 0)
        {
            nrun = r;
            rgroups = f.y;
            break;
        }
    }
    long long pos = sizes ? 0 : off[so];
    const int half = threadIdx.x >> 6, e = threadIdx.x & 63;
    for (int r = 0; r < nrun; r++)
    {
        const int g0 = fl[r].y, g1 = r + 1 < nrun ? fl[r + 1].y : rgroups;
        for (int cg = g0; cg < g1; cg += GMAX)
        {
            const int nent = UPGEO_RUN * min(GMAX, g1 - cg);
            const int N = (nent + 15) & ~15;
            if (!sizes && e < N)
            {
                UpGeo32 g;
                g.node = -1;
                g.loc[0] = g.loc[1] = g.loc[2] = 0.f;
                g.tr = g.ti = 0.f;
                if (e < nent)
                    g = geo32[(slot * 8 + o) * P_pad + (size_t)(e % UPGEO_RUN) * ngroups + cg +
                              e / UPGEO_RUN];
                const int node = e < nent ? g.node : -1;
                int4* meta = reinterpret_cast<int4*>(img + pos);
                float* B = reinterpret_cast<float*>(img + pos + 16 * N);
                float* bh = B + (size_t)(e >> 3) * (S::SBO / 4) + (e & 7) * 4;
                float* bl = B + (size_t)((N + e) >> 3) * (S::SBO / 4) + ((N + e) & 7) * 4;
                if (half == 0)
                {
                    if (!meta_only)
                        uptc_basis_half<N0, N1, N2, 0>(node >= 0, g.loc[0], g.loc[1], g.loc[2], bh,
                                                       bl);
                    meta[e] = make_int4(node, __float_as_int(g.tr), __float_as_int(g.ti), 0);
                }
                else if (!meta_only)
                    uptc_basis_half<N0, N1, N2, 1>(node >= 0, g.loc[0], g.loc[1], g.loc[2], bh, bl);
            }
            pos += (long long)N * (16 + 8 * K);
        }
    }
    if (sizes && threadIdx.x == 0)
        sizes[so] = pos;
}

// Order shapes with a tensor-core upward kernel: the low orders of p = 8 and
// p = 9 (an even number of coefficients, at most 128 of them).
template <int N0, int N1, int N2> constexpr bool uptc_shape()
{
    return (N0 == 2 && N1 == 5 && N2 == 5) || (N0 == 3 && N1 == 6 && N2 == 6);
}

// Launches the tensor-core upward transfer of one level over `n_tiles` row
// tiles (a.tc_tiles) when the path, the order shape, the tile fill and the
// shared memory allow; returns false (nothing launched) otherwise, and the
// caller runs an FFMA kernel.
// choice: the autotuner's decision for this level and plane count (1 tensor
// cores, 0 FFMA), or -1 when there is none (AUTO then falls back to the tile
// fill).
template <int KIND, int N0, int N1, int N2>
bool launch_upward_tc(const UpArgs& a, int n_tiles, float fill, int path, cudaStream_t st,
                      int planes = 1, int choice = -1)
{
    if constexpr (!uptc_shape<N0, N1, N2>())
        return false;
    else
    {
        if (path == UP_FFMA || !a.tc_tiles || n_tiles <= 0 || !a.tc_status || a.kp_plane ||
            a.fe_pad <= 0)
            return false;
        if (path == UP_AUTO && (choice == 0 || (choice < 0 && fill < UPTC_MIN_FILL)))
            return false;
        // 16-byte aligned coefficient planes for the bulk copies
        if (planes > 1 && (a.fc_plane % 2) != 0)
            return false;
        const size_t sm = uptc_smem_bytes<N0, N1, N2>(a.P_hi, a.fe_pad);
        if (sm > 227 * 1024)
            return false;
        auto kern = upward_tc_kernel<KIND, N0, N1, N2>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sm);
        if (e != cudaSuccess)
            throw Error(2, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        kern<<<n_tiles, UPTC_THREADS, sm, st>>>(a);
        return true;
    }
}

} // namespace ifgf
