// Launch interface of the matvec kernels (implemented in mult_kernels.cuh,
// instantiated once per kernel plug-in in kernels_k<KIND>.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.hpp"
#include "device_math.cuh"

namespace ifgf
{

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

// Box-independent geometry of the upward transfer at one level: for parent
// cone element slot s, octant o and Chebyshev node n of the parent cone, the
// child's fine element (or -1 when the node lies outside the child's
// interpolation domain), the node's local coordinates in that element and
// the centre-shift factor G(y, x_child)/G(y, x_parent).
// Each (slot, octant) row is sorted by child element, so that the threads of
// a warp gather the same cone's coefficients; `node` is the parent node the
// entry belongs to.
// 16-byte aligned, so that an entry loads as whole 16-byte vectors (a
// warp reading consecutive entries touches each sector once, not once per
// field)
struct __align__(16) UpGeo64
{
    double loc[3];
    double tr, ti;
    int fe;
    int node;
};
struct __align__(16) UpGeo32
{
    float loc[3];
    float tr, ti;
    int fe;
    int node;
    int pad;
};
static_assert(sizeof(UpGeo64) == 48 && sizeof(UpGeo32) == 32, "table entry sizes");

// Per-level device lists of one operator.
struct LevelLists
{
    const int* cc_box;   // coarse cone -> global box id
    const int* cc_el;    // coarse cone -> element id
    const int* leaf_idx; // coarse cones of leaf boxes (indices into cc_*)
    const int* up_idx;   // coarse cones of boxes with children, ordered by element
    const int* up_slot;  // element slot of each up_idx entry (geometry table row)
    const UpGeo64* geo64; // [slot][octant][up_pad entries]
    const UpGeo32* geo32;
    int n_leaf, n_up;
    int up_pad; // row stride of the geometry tables
    const int2* fe_list; // [slot][octant][fe_pad + 1]: (child element, first group) of each
                         // run, then (-1, groups of the row)
    int fe_pad;         // longest run list of a row
    const int* c2f_idx; // coarse cones to refine when n_c2f >= 0 (sharded operators)
    int n_c2f;          // -1: all of the level's cones
    // tensor-core upward transfer of single-plane matvecs: row tiles (first
    // up_idx position, cones, first plane, planes) and the fraction of their
    // 32 rows that hold cones
    const int4* tc_tiles = nullptr;
    int n_tc_tiles = 0;
    float tc_fill = 0.f;
    // basis images of the tensor-core upward transfer (null: none), with the
    // byte offset of every (slot, octant)
    const unsigned char* tc_img = nullptr;
    const long long* tc_img_off = nullptr;
};

// Upward-transfer kernel choice (Operator::set_upward_path): AUTO takes the
// tensor-core kernel on levels whose row tiles are at least UPTC_MIN_FILL
// full, FFMA never, TENSOR wherever the order shape and shared memory allow.
enum UpwardPath : int
{
    UP_AUTO = 0,
    UP_FFMA = 1,
    UP_TENSOR = 2
};
constexpr float UPTC_MIN_FILL = 0.4f;

// Upward geometry tables of one level, built on the device in two passes:
// upgeo_row_max measures every (slot, octant) row's padded length and number
// of element runs (row_len scratch of 16 n_slots ints) and returns the
// longest row, the row stride P_pad, with the most runs of a row in
// *runs_max; launch_build_upgeo fills tables pre-set to all-ones bytes
// (skipped entries) and the per-row element lists (fe_pad entries a row,
// pre-set to -1).  slot_el: element id of each slot; off: 8 child-centre
// offsets.  With g64 null it fills g32 as a distance table (tr = d - d_parent,
// ti = d_parent / d) for multi-wavenumber batches.
template <int KIND>
int upgeo_row_max(const LevelGeom& PG, const LevelGeom& CG, double pH, double cH,
                  const double* off_dev, const int* slot_el, int n_slots, const double* hi_nodes,
                  int P_hi, KParams kp, int* row_len_dev, int* row_len_host, int* runs_max);
template <int KIND>
void launch_build_upgeo(const LevelGeom& PG, const LevelGeom& CG, double pH, double cH,
                        const double* off_dev, const int* slot_el, int n_slots,
                        const double* hi_nodes, int P_hi, KParams kp, int P_pad, UpGeo64* g64,
                        UpGeo32* g32, int fe_pad, int2* fe_list);

// Everything one matvec launch needs (device pointers, sizes, orders).
struct MultPtrs
{
    int L;
    const LevelGeom* lv_host; // host copy (grid sizes)
    const LevelGeom* lv_dev;  // device copy (read by target_eval)
    const LevelLists* lists;  // host array of L entries
    TreeArgs T;
    SrcArgs S;
    const double* tx;
    const double* ty;
    const double* tz;
    const long long* src_perm;
    const long long* tgt_perm;
    const double* hi_nodes;
    const double* A;
    const double* A_host; // host copy of A (fixed-order kernels take it by value)
    const int* fmap;
    const int* tl_first;
    const int* tl_last;
    const long long* tl_far_off;
    const int* tl_far_src;
    const long long* tl_near_off;
    const int* tl_near_src;
    int n_tleaf;
    long long n_src;
    double2* w;
    double2* cvals;
    double2* fcoef;
    double2* unear; // near-field sums per sorted target
    unsigned long long* err;
    // second stream for the near field, which overlaps the level loop
    cudaStream_t side;
    cudaEvent_t ev_fork, ev_join;
    int lo[3], hi[3], fct[3];
    int P_lo, P_hi;
    size_t c2f_smem; // for FP64 buffers (half of it in mixed precision)
    KParams kp;
    bool mixed; // mixed-precision pipeline (buffers hold float2)
    int up_path = UP_AUTO;           // UpwardPath
    unsigned* tc_status = nullptr;   // bounded-wait status of the tensor-core kernels
    // the upward-kernel autotuner's per-level choice for single-plane
    // matvecs (host array of L: 1 tensor cores, 0 FFMA, -1 none yet)
    const signed char* up_choice = nullptr;
};



// Stage classes for per-kernel timing.
enum ProfClass
{
    PROF_PERMUTE = 0,
    PROF_COARSE = 1, // leaf sampling
    PROF_C2F = 2,
    PROF_EVAL = 3, // far field (+ the near sums)
    PROF_UPWARD = 4,
    PROF_NEAR = 5
};

struct LaunchHooks
{
    // cls: ProfClass; level: source-tree level of a per-level launch, else -1
    virtual void begin(int cls, int level = -1) = 0;
    virtual void end() = 0;
    virtual ~LaunchHooks() = default;
};

// Enqueues one matvec on `st`; returns the number of kernels launched.
template <int KIND>
int launch_mult_kernels(const MultPtrs& m, const void* d_w, void* d_u, bool real, cudaStream_t st,
                        LaunchHooks* hooks);

// Planes of the batched mixed matvec (mult_batch.cuh): a launch covers
// `groups` groups of BATCH_NB planes; plane p (group p / BATCH_NB) lives at
// offset p * plane of each buffer.
constexpr int BATCH_NB = 4;
// Far-field plan of the batched mixed matvec (built once per init, used by
// every batched or multi-wavenumber matvec): the (target, far box) pairs of
// each target-leaf chunk in groups of S consecutive far boxes (one pair per
// thread of a 256-thread CTA, thread = target + (box - first box) x targets),
// each group's distinct fine cones in slots (the 24 with the most pairs)
// and its pairs as records in slot order, every slot's run padded to
// FAR_PLAN_PAD positions (4: a quad of evaluating lanes takes 8, so about
// half the quads of a slot's last positions straddle two slots and read two
// blocks -- measured cheaper than padding to 8, which evaluated some 30 %
// padding positions, or to 2).
struct FarChunk // up to 256 targets of one target leaf
{
    long long g0, g1; // its groups
    int t0, cnt;      // first target (sorted order) and number of targets
};
struct FarGroup
{
    long long rec;  // first record
    long long box0; // index of its first far box in the target-leaf far list
    int slot;       // first slot cone id (then the cone ids of its overflow records)
    unsigned short npos, nslotted; // records: all, in slots (padded)
    unsigned short nbox;           // boxes in the group
    unsigned char nslot;           // slots
    unsigned char pad_;
};
// local coordinates (float bits) and w = owner thread | slot << 9 (slot 31:
// read from global memory, cone id in the group's overflow list; owner 511:
// padding)
struct __align__(16) FarPlanRec
{
    int l0, l1, l2, w;
};
// slots per group of a plan: FAR_PLAN_SLOTS, or the larger of
// FAR_PLAN_SLOTS_MID and FAR_PLAN_SLOTS_FEW that lets more far CTAs reside
// per SM, where at most 3 % of the records then read global memory
constexpr int FAR_PLAN_SLOTS = 24;
constexpr int FAR_PLAN_SLOTS_MID = 18;
constexpr int FAR_PLAN_SLOTS_FEW = 16;
constexpr int FAR_PLAN_THREADS = 256, FAR_PLAN_PAD = 4;
// record positions of a group with nsl slots (each slot's run padded)
__host__ __device__ constexpr int far_plan_pos(int nsl)
{
    return (FAR_PLAN_THREADS + (FAR_PLAN_PAD - 1) * nsl + 7) / 8 * 8;
}
// float2 per shared-memory slot of np planes of p_lo coefficients, padded
// to start 16 bytes apart modulo 128
__host__ __device__ constexpr int far_slot_stride_rt(int p_lo, int np)
{
    int s = np * p_lo;
    while ((s * 8) % 128 != 16 && (s * 8) % 128 != 80)
        s++;
    return s;
}
// resident CTAs per SM of the plan's far kernel with nsl slots: as many as
// its shared memory allows (slots, records, values, factors, 1 KB reserved
// per CTA), at most three (80 registers a thread; two get 128)
__host__ __device__ constexpr int far_plan_ctas(int nsl, int p_lo, int np)
{
    const int bytes = nsl * far_slot_stride_rt(p_lo, np) * 8 + far_plan_pos(nsl) * 16 +
                      np * (FAR_PLAN_THREADS + 1) * 8 + np * (int)sizeof(KParams) + 1024 + 512;
    const int n = 233472 / bytes;
    return n < 1 ? 1 : (n > 3 ? 3 : n);
}
constexpr int FAR_PLAN_OVF = 31;
constexpr int FAR_PLAN_PAD_OWNER = 511;

struct BatchPtrs
{
    float2* w;      // planes of n_src permuted densities
    float2* cvals;  // planes of cv_plane coarse values
    float2* fcoef;  // planes of fc_plane fine coefficients
    double2* unear; // planes of n_tgt near-field sums
    long long cv_plane, fc_plane;
    long long n_src, n_tgt;
    int nrhs;                      // planes holding right-hand sides (the rest are zero)
    int groups = 1;                // plane groups in one launch (nrhs <= groups * BATCH_NB)
    long long in_plane, out_plane; // caller's density / result strides (in doubles)
    // wavenumber of every plane (device, groups * BATCH_NB entries), or null
    // when all planes share the operator's; with it the upward transfer reads
    // the distance tables (UpGeo32::tr = d - d_parent, ::ti = d_parent / d)
    const KParams* kp_plane = nullptr;
    const UpGeo32* const* dgeo32 = nullptr; // per level (host array)
    // tensor-core upward tiles for groups * BATCH_NB planes, per level (host
    // arrays; null: FFMA kernel)
    const int4* const* tc_tiles = nullptr;
    const int* n_tc_tiles = nullptr;
    const float* tc_fill = nullptr;
    const signed char* up_choice = nullptr; // autotuner's choice for these planes (per level)
    // far-field plan (null: the far kernel finds cones and slots itself)
    const FarChunk* fp_chunk = nullptr;
    int fp_nchunk = 0;
    int fp_nslot = 0; // slots per group the plan was built for
    const FarGroup* fp_group = nullptr;
    const FarPlanRec* fp_rec = nullptr;
    const int* fp_slot = nullptr;
};

// Basis images of the tensor-core upward transfer of one level, for the low
// order shape lo (a shape with a tensor-core kernel): for every (slot,
// octant) row of the geometry tables and every chunk of <= 48 entries of its
// runs (the walk of the kernel), the chunk's entry data (node, centre-shift
// factor) and its B operand -- the TF32 high and low parts of the basis rows
// in the kernel's shared-memory layout -- so that the kernel copies them
// instead of computing them in every tile of the slot.
// upward_tc_image_sizes writes the bytes of every row (nslots x 8 entries);
// upward_tc_image_fill writes the images at the given byte offsets (with
// meta_only, just the entry data: after the wavenumber changed).
// Both synchronise the device.  False: no tensor-core kernel for lo.
// Levels get images when their slots average at least UPTC_IMG_MIN_CONES
// cones (row tiles reusing each image), up to UPTC_IMG_BUDGET bytes in all.
constexpr double UPTC_IMG_MIN_CONES = 24.0;
constexpr long long UPTC_IMG_BUDGET = 8ll << 30;
bool upward_tc_image_sizes(const int* lo, const int2* fe_list, int fe_pad, int up_pad, int nslots,
                           long long* d_sizes);
bool upward_tc_image_fill(const int* lo, const int2* fe_list, int fe_pad, const UpGeo32* geo32,
                          int up_pad, int nslots, const long long* d_off, unsigned char* img,
                          bool meta_only = false);

// Enqueues the mixed matvec of bp.nrhs <= bp.groups * BATCH_NB right-hand
// sides, one launch per stage and level for all of them; planes of a group
// share the kernel and geometry work (with kp_plane: the geometry only).
// Returns the kernels launched, or -1 when the operator's orders or upward
// rows have no batched path.
template <int KIND>
int launch_mult_batch_kernels(const MultPtrs& m, const BatchPtrs& bp, const void* d_w, void* d_u,
                              bool real, cudaStream_t st, LaunchHooks* hooks);

// Upward-kernel autotuner: for every level whose shape has both kernels,
// the FFMA and the tensor-core upward transfer of one launch over `planes`
// right-hand-side planes (bp null: the single-plane buffers of m) are timed
// on the operator's own tables and buffers (each kernel once to warm up,
// then the better of two timed launches); choice[l] = 1 where the tensor
// cores were faster by more than 3 %, 0 elsewhere, -1 on levels without
// both kernels; ms_ffma / ms_tc receive the times (0 where not timed).
// The buffers' contents are left unspecified (the next matvec rewrites
// them).  Returns the number of levels timed.
template <int KIND>
int tune_upward_kernels(const MultPtrs& m, const BatchPtrs* bp, int planes, cudaStream_t st,
                        signed char* choice, double* ms_ffma, double* ms_tc);

// Only the density permutation into m.w (for direct sums).
template <int KIND>
void permute_only(const MultPtrs& m, const void* d_w, bool real, cudaStream_t st);

// FP64 direct sums at the sorted target positions tpos[0..nt) (weights must
// already be permuted into m.w).
template <int KIND>
void launch_direct_kernel(const MultPtrs& m, const int* tpos, int nt, double2* out,
                          cudaStream_t st);

// Order estimation probe (ifgfoperator.hpp:204-212): the factored kernel of
// a sample box's sources with unit weights at Cartesian nodes.  Sample s owns
// sources [src_off[s], src_off[s + 1]) of S and nodes [node_off[s],
// node_off[s + 1]) of `nodes` (xyz triples); out receives one value per node.
struct ProbeArgs
{
    SrcArgs S;
    const int* __restrict__ src_off;
    const double* __restrict__ nodes;
    const int* __restrict__ node_off;
    const double* __restrict__ centre; // 3 per sample
    KParams kp;
    double2* out;
};

template <int KIND>
void launch_order_probe(const ProbeArgs& a, int n_samples, int max_nodes, cudaStream_t st);

} // namespace ifgf
