// The IFGF operator object behind the C ABI: host planner + device tables +
// the per-level CUDA pipeline.  No CUDA types appear in this header.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "common.hpp"
#include "plan.hpp"

namespace ifgf
{

struct DeviceState;  // device buffers, defined in operator.cu
struct MultPtrs;     // kernel launch view, defined in mult.hpp
struct AdjointState; // operators and buffers of the adjoint, defined in operator.cu
struct EventHooks;   // per-launch CUDA events, defined in operator.cu
struct BatchPtrs;    // plane buffers of the batched pipeline, mult.hpp

struct StageTimes
{
    double permute = 0, coarse = 0, c2f = 0, eval = 0, upward = 0, near = 0, total = 0;
};

class Operator
{
  public:
    // IfgfOperator ctor (ifgfoperator.hpp:36-59) + plug-in ctor
    Operator(int kind, double k_re, double k_im, int64_t leaf_size, int64_t order, int64_t n_elem,
             double tol);
    ~Operator();

    void set_dx(int dx);
    // Change the wavenumber of an initialised operator.  When every level's
    // cone grids stay the same (elementsForBox), the tree, lists and cone
    // maps are kept and only the k-dependent centre-shift factors of the
    // upward geometry are recomputed; otherwise the operator is initialised
    // again from the points of the last init.  Frequency sets (convolution
    // quadrature) thus share one tree and one set of cone maps.
    void set_wavenumber(double k_re, double k_im);
    // Take share `rank` of `nranks` of the matvec (before init): mult then
    // returns the contribution of this rank's source subtrees to every
    // target, and the ranks' results sum to the full matvec (see
    // Plan::assign_shards).
    void set_shard(int rank, int nranks);
    // recursive level of the shards and this rank's boxes on it
    int shard_level() const { return plan_.shard_level; }
    std::vector<int64_t> shard_boxes() const;
    void set_precision(int mode);
    // IfgfOperator::init (ifgfoperator.hpp:65-106)
    void init(const double* srcs, int64_t ns, const double* tgts, int64_t nt,
              const double* normals, const std::function<bool(double)>& cutoff,
              bool plan_only = false);
    // IfgfOperator::mult on device buffers; stream is a cudaStream_t
    void mult_device(const void* d_w, void* d_u, void* stream);
    // host buffers, `batch` right-hand sides
    void mult_host(const void* w, void* u, int64_t batch);
    // `batch` right-hand sides on device buffers (batch x n_src in, batch x
    // n_tgt out).  The mixed pipeline runs them through the batched kernels,
    // one launch per stage and level for up to 64 right-hand sides (groups of
    // BATCH_NB share one kernel / geometry evaluation); FP64 and shapes
    // without a batched path run them one by one.
    void mult_batch_device(const void* d_w, void* d_u, int64_t batch, void* stream);
    // Multi-wavenumber batch: right-hand side p (plane p of d_w / d_u) is
    // multiplied at wavenumber k[2p] + i k[2p+1].  Every wavenumber must give
    // the operator's cone grids (a convolution-quadrature set does); the
    // planes share the tree, cone maps and geometry of one pass, one launch
    // per stage and level for up to 64 planes (mixed precision).  FP64 runs
    // one set_wavenumber refresh and matvec per plane.
    void mult_wavenumbers_device(const double* k, int64_t nk, const void* d_w, void* d_u,
                                 void* stream);
    // the same with host buffers
    void mult_wavenumbers_host(const double* k, int64_t nk, const void* w, void* u);
    // mult_device with its scratch in a caller-provided device region instead
    // of the buffers allocated at init; allocates nothing
    void mult_device_external_scratch(const void* d_w, void* d_u, void* stream, void* scratch,
                                      size_t scratch_bytes);
    // (dA/dk) w for the Helmholtz and combined-field kernels: the same tree,
    // cones and orders, with the k-derivative kernel (K_HELMHOLTZ_DK,
    // K_COMBINEDFIELD_DK); its upward geometry is tabulated on first use
    void mult_dk_device(const void* d_w, void* d_u, void* stream);
    void mult_dk_host(const void* w, void* u, int64_t batch);
    // kernel of the k-derivative, or -1 when the kernel has none
    int dk_kind() const;
    // u = A^H w (w over the targets, u over the sources).  Kernels symmetric
    // under exchanging source and target (Laplace, Helmholtz, modified
    // Helmholtz) give conj(A' conj(w)) with A' the operator with the roles of
    // the point sets swapped (A itself when sources and targets are the same
    // points); the gradient kernel, antisymmetric, the negative of that; the
    // double-layer and combined-field kernels carry the normal at the new
    // target and are composed from three swapped gradient operators (plus a
    // swapped Helmholtz one for the combined field).  The operators are built
    // on first use from the points, normals and cutoff of init.
    void mult_adjoint_device(const void* d_w, void* d_u, void* stream);
    void mult_adjoint_host(const void* w, void* u, int64_t batch);
    // FP64 direct sum at selected targets (original indices), host buffers;
    // with dk, of the k-derivative kernel
    void direct_eval(const void* w, const int64_t* tidx, int64_t nt, void* out, bool dk = false);
    void set_profiling(bool on);
    // upward-transfer kernel: UP_AUTO, UP_FFMA or UP_TENSOR (mult.hpp)
    void set_upward_path(int path);
    void set_far_plan(bool on);
    bool far_plan() const { return far_plan_on_; }
    int upward_path() const { return up_path_; }
    // throws IFGF_ERR_TIMEOUT when a tensor-core kernel's bounded wait gave up
    void check_device_status();

    int kind() const { return kind_; }
    bool is_real() const { return kind_ == K_LAPLACE; }
    int64_t n_src() const { return plan_.src.n; }
    int64_t n_tgt() const { return plan_.tgt.n; }
    bool initialized() const { return initialized_; }
    bool planned() const { return planned_; }
    const Plan& plan() const { return plan_; }
    void orders(int step, int* o) const;
    void level_grid(int level, int step, int64_t* n) const;
    std::vector<int64_t> box_cones(int level, int64_t box, int step) const;
    std::string stats_json() const;

  private:
    void order_for_box(int step, int* out) const;
    void elements_for_box(double H, int step, int64_t* out) const;
    double cutoff_limit(double H) const;
    void set_orders();
    void estimate_orders(int* out) const;
    bool grids_match(double k_re, double k_im);
    int ensure_batch_planes(int64_t want);
    BatchPtrs batch_ptrs(long long in_plane, long long out_plane) const;
    void ensure_distance_tables();
    void ensure_tc_tiles(int planes);
    void set_batch_tc(BatchPtrs& bp, void* stream);
    // far-field plan of the batched mixed matvec: built on first use (once
    // per init), handed to the far kernel through bp; off: the far kernel
    // finds its cones itself (no plan memory)
    void ensure_far_plan();
    void set_batch_far(BatchPtrs& bp);
    void ensure_upward_tuned(int planes, const BatchPtrs* bp, void* stream);
    // basis images of the tensor-core upward transfer (built on first use of
    // the mixed pipeline; their entry data is rewritten by set_wavenumber)
    void ensure_tc_images();
    void setup_device(const double* normals);
    // vkind >= 0: run that kernel with the variant geometry tables
    void launch_mult(const void* d_w, void* d_u, void* stream, bool timed, int vkind = -1);
    void fill_mult_ptrs(MultPtrs& m, bool variant = false) const;
    void ensure_variant_tables(int vkind);
    void ensure_adjoint();
    void finish_profile(EventHooks& log, int rhs);
    void host_mult_loop(const void* w, void* u, int64_t batch, int vkind);

    int kind_;
    double kr_, ki_;
    int dx_ = -1;
    double tol_;
    int64_t leaf_;
    int order0_;
    int base_order_[3];
    int64_t base_n_[3];
    int precision_ = PREC_FP64;
    int device_ = -1; // CUDA device of the device tables (set by init)
    int up_path_ = 0; // UpwardPath
    bool far_plan_on_ = true;
    bool initialized_ = false;
    bool planned_ = false;
    Plan plan_;
    std::vector<LevelGeom> lv_;
    int lo_[3], hi_[3];
    int fct_[3];
    std::unique_ptr<DeviceState> dev_;
    // init inputs in the caller's order, kept for the adjoint operators
    std::vector<double> src_pts_, tgt_pts_, normals_;
    std::function<bool(double)> cutoff_;
    bool same_points_ = false;
    std::unique_ptr<AdjointState> adj_;
    int shard_rank_ = 0, shard_n_ = 1;
    // statistics
    double init_ms_ = 0, tree_ms_ = 0, lists_ms_ = 0, tlists_ms_ = 0, device_ms_ = 0;
    std::vector<std::pair<std::string, double>> dev_phases_; // setup_device phases (ms)
    StageTimes last_;
    int64_t n_coarse_total_ = 0, n_fine_total_ = 0;
    double leaf_evals_ = 0, upward_evals_ = 0;
    double upgeo_bytes_ = 0; // device bytes of the upward geometry tables
    std::vector<int> fe_pad_; // per level: most element runs in one upward geometry row
    struct UpwardLevelStats
    {
        int64_t cones = 0, slots = 0, blocks = 0, entries = 0;
    };
    std::vector<UpwardLevelStats> up_stats_;
    unsigned long long missing_ = 0;
    bool profiling_ = false;
    // per kernel class: launches and accumulated milliseconds
    // permute, leaf_sample, coarse_to_fine, target_eval, upward
    static constexpr int NPROF = 6;
    int64_t prof_launches_[NPROF] = {};
    double prof_ms_[NPROF] = {};
    double prof_level_ms_[NPROF][MAX_LEVELS] = {}; // per-level launches only
    int64_t mults_profiled_ = 0;
    int launches_per_mult_ = 0;
};

} // namespace ifgf
