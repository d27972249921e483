/*
 * ifgf_b200 -- C ABI of the B200 IFGF matvec library (libifgf_b200.so).
 *
 * The entry points below are the boundary a foreign-function binding of the
 * reference's operator would bind.  The reference exposes its operators
 * through pybind11 (py_ifgf.cpp:16-58); each function names the reference
 * interface it replaces.  Plain pointers and sizes only; every call returns an
 * int status (IFGF_OK == 0) and ifgf_last_error() gives a message for the
 * calling thread's last failure.
 *
 * Point arrays are float64, 3 x N in column-major order (x0,y0,z0,x1,...),
 * the memory layout of the reference's Eigen::Array<double, 3, Dynamic>.
 * Densities and results are complex128 (interleaved re, im) for every kernel
 * except Laplace, whose densities and results are float64 (the reference's
 * T = double, laplace_ifgf.hpp:8).
 *
 * A handle owns all of its device memory.  Calls on one handle are not
 * thread-safe; separate handles are independent.
 */
#ifndef IFGF_B200_H
#define IFGF_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ifgf_operator ifgf_operator;

/* status codes */
#define IFGF_OK 0
#define IFGF_ERR_INVALID_ARG 1 /* bad size, order, kind, NaN/Inf input, ... */
#define IFGF_ERR_CUDA 2        /* a CUDA runtime call failed                  */
#define IFGF_ERR_STATE 3       /* e.g. mult before init                      */
#define IFGF_ERR_OOM 4         /* device allocation failed                   */
#define IFGF_ERR_TIMEOUT 5     /* a bounded device wait gave up              */
#define IFGF_ERR_INTERNAL 6    /* consistency check failed (cone lookups)    */

/* kernel plug-ins (one per reference Derived class) */
#define IFGF_LAPLACE 0            /* laplace_ifgf.hpp                    */
#define IFGF_HELMHOLTZ 1          /* helmholtz_ifgf.hpp                  */
#define IFGF_MODIFIED_HELMHOLTZ 2 /* modified_helmholtz_ifgf.hpp         */
#define IFGF_GRAD_HELMHOLTZ 3     /* grad_helmholtz_ifgf.hpp             */
#define IFGF_DOUBLE_LAYER 4       /* double_layer_helmholtz_ifgf.hpp     */
#define IFGF_COMBINED_FIELD 5     /* combined_field_helmholtz_ifgf.hpp   */

/* precision modes */
#define IFGF_PREC_FP64 0  /* FP64 throughout                                  */
#define IFGF_PREC_MIXED 1 /* FP32 sums with FP64 phase / final accumulation   */

/* ifgf_set_upward_path */
#define IFGF_UPWARD_AUTO 0   /* per level, the faster of the two (timed)      */
#define IFGF_UPWARD_FFMA 1   /* FP32 FMA kernels only                         */
#define IFGF_UPWARD_TENSOR 2 /* tensor cores wherever the order shape allows  */

/* Replaces the IfgfOperator constructor (ifgfoperator.hpp:36-59) together
 * with the plug-in constructors (helmholtz_ifgf.hpp:13-20,
 * laplace_ifgf.hpp:12-15, modified_helmholtz_ifgf.hpp:13-20,
 * grad_helmholtz_ifgf.hpp:13-21, double_layer_helmholtz_ifgf.hpp:13-20,
 * combined_field_helmholtz_ifgf.hpp:13-20) as bound at py_ifgf.cpp:19, :46.
 * k = k_re + i k_im is the wavenumber (ignored by Laplace; the imaginary part
 * is ignored by the real-wavenumber Helmholtz and combined-field kernels).
 * tol <= 0 selects the fixed orders (max(order - 3, 2), order, order)
 * (ifgfoperator.hpp:88-91).  tol > 0 makes ifgf_init estimate the orders
 * (estimateRefinement, ifgfoperator.hpp:80-85, 108-244: ten boxes of the
 * deepest source level, kernel samples on the GPU) and also sets the gradient
 * kernel's cutoff (grad_helmholtz_ifgf.hpp:294-304); ifgf_orders reports
 * the result.  A plan-only init refuses tol > 0. */
int ifgf_create(int kind, double k_re, double k_im, long leaf_size, long order, long n_elem,
                double tol, ifgf_operator** out);

/* Replaces GradHelmholtzIfgfOperator::setDx (grad_helmholtz_ifgf.hpp:61,
 * py_ifgf.cpp:40): dx in {-1, 0, 1, 2}. */
int ifgf_set_dx(ifgf_operator* op, int dx);

/* Changes the wavenumber of an operator.  After init, when the new k gives
 * every level the same cone grids (elementsForBox of the kernel), the tree,
 * interaction lists and active-cone maps are kept and only the k-dependent
 * centre-shift factors are recomputed (milliseconds); otherwise the operator
 * is initialised again from the points, normals and cutoff of its last init.
 * For frequency sets (convolution quadrature), where the reference builds a
 * new operator per frequency (test/test_CQIFGF.cpp:117-135). */
int ifgf_set_wavenumber(ifgf_operator* op, double k_re, double k_im);

/* Selects FP64 (default) or the mixed-precision pipeline.  No reference
 * counterpart (the reference is FP64 only). */
int ifgf_set_precision(ifgf_operator* op, int mode);

/* Selects the kernel of the mixed-precision upward transfer (the
 * interpolation of children's fine interpolants at parent cone nodes,
 * transferInterp, ifgfoperator.hpp:1639-1705): IFGF_UPWARD_AUTO (default)
 * times the tensor-core kernel (tcgen05, split-TF32, FP32-accurate) and the
 * FP32 FMA kernel once per level and right-hand-side count on the operator's
 * own tables (the first mixed matvec of that count) and keeps the faster per
 * level (the choice and the times are in ifgf_stats_json, "upward_tuner");
 * levels it has not timed use the tensor cores when their cones fill the
 * kernel's 32-row tiles well enough; IFGF_UPWARD_FFMA never uses the tensor cores;
 * IFGF_UPWARD_TENSOR uses them on every level the order shape allows (low
 * orders (2,5,5) and (3,6,6)).  FP64 always runs the FP64 kernels.  No
 * reference counterpart. */
int ifgf_set_upward_path(ifgf_operator* op, int path);

/* Far-field plan of the batched and multi-wavenumber mixed matvecs
 * (enable = 1, the default): on their first call the (target, far box) pairs
 * of every target leaf are looked up once -- fine cone, local coordinates --
 * and stored grouped and sorted by cone (a 16-byte record per pair plus
 * padding, about 19 bytes per pair in all: 7.2 GB at N = 1e6, k = 100, p = 9;
 * the size is in ifgf_stats_json, "far_plan"),
 * so that every later matvec skips the lookups (evaluateFromInterp,
 * ifgfoperator.hpp:1736-1891, done as a lookup pass at setup and a sum pass
 * per matvec).  enable = 0 frees the plan and the far kernel looks the cones
 * up in every matvec (same results).  No reference counterpart. */
int ifgf_set_far_plan(ifgf_operator* op, int enable);

/* Diagnostic of the bounded waits the tensor-core kernels use: launches a
 * one-block kernel that waits, for at most limit_ms milliseconds, on a
 * barrier that nothing arrives at.  Returns IFGF_ERR_TIMEOUT (the wait gave
 * up and the kernel returned normally, as designed) with the time the kernel
 * waited in *waited_ms; any other status means the mechanism is broken.  No
 * reference counterpart. */
int ifgf_bounded_wait_selftest(double limit_ms, double* waited_ms);

/* Multi-GPU sharding, called before ifgf_init: the operator takes share
 * `rank` of `nranks` -- a contiguous Morton range, balanced by modelled work,
 * of the source subtrees rooted at the first level that has far pairs (no
 * box above it has far targets, so the subtrees are independent).  Its
 * matvec returns the contribution of those subtrees to every target, and the
 * ranks' results sum to the full matvec (one all-reduce of n_tgt values).
 * Each rank builds the whole tree and cone maps.  No reference counterpart:
 * the reference runs those subtrees as parallel tasks on one host
 * (ifgfoperator.hpp:330-340). */
int ifgf_set_shard(ifgf_operator* op, int rank, int nranks);

/* After init: the shard level and this rank's boxes on it (level-local box
 * indices, *n of them, at most cap written).  No reference counterpart. */
int ifgf_shard_boxes(const ifgf_operator* op, int* level, long* boxes, long cap, long* n);

/* Far-interaction drop predicate of IfgfOperator::init
 * (ifgfoperator.hpp:65-67, octree.hpp:282-297): return nonzero to drop an
 * admissible pair at exterior distance `dist`.  May be NULL. */
typedef int (*ifgf_cutoff_fn)(double dist, void* user);

/* Replaces IfgfOperator::init (ifgfoperator.hpp:65-106) and the double-layer
 * / combined-field init(srcs, targets, normals)
 * (double_layer_helmholtz_ifgf.hpp:22-26,
 * combined_field_helmholtz_ifgf.hpp:22-26).  normals: 3 x n_src, required for
 * IFGF_DOUBLE_LAYER and IFGF_COMBINED_FIELD, ignored otherwise. */
int ifgf_init(ifgf_operator* op, const double* srcs, long n_src, const double* tgts,
              long n_tgt, const double* normals, ifgf_cutoff_fn cutoff, void* user);

/* Host half of ifgf_init: builds the octrees and interaction lists only,
 * touching no GPU (the tree and list accessors below work after it; mult
 * does not).  For tests and tooling on machines without a GPU.  Replaces the
 * first steps of IfgfOperator::init, Octree::build of both point sets and
 * buildInteractionList (ifgfoperator.hpp:69-72). */
int ifgf_init_plan_only(ifgf_operator* op, const double* srcs, long n_src, const double* tgts,
                        long n_tgt, ifgf_cutoff_fn cutoff, void* user);

/* Replaces IfgfOperator::mult (ifgfoperator.hpp:246-867) with host buffers:
 * w has n_src entries, u receives n_tgt entries (caller's original order). */
int ifgf_mult(ifgf_operator* op, const void* w, void* u);

/* Same as ifgf_mult for `batch` right-hand sides stored one after another
 * (w: batch x n_src, u: batch x n_tgt).  In the mixed-precision pipeline the
 * right-hand sides run through batched kernels, one launch per stage and
 * level for up to 64 of them; groups of four share the kernel, cone-lookup
 * and centred-factor evaluations (each right-hand side keeps its own
 * interpolants); FP64 runs them one by one.  No reference counterpart. */
int ifgf_mult_batch(ifgf_operator* op, const void* w, void* u, long batch);

/* ifgf_mult_batch on device buffers enqueued on `stream`.  No reference
 * counterpart. */
int ifgf_mult_batch_device(ifgf_operator* op, const void* d_w, void* d_u, long batch,
                           void* stream);

/* Multi-wavenumber batch: u_p = A(k_p) w_p for p < n_k, with
 * k_p = k[2p] + i k[2p+1] and w / u stored as in ifgf_mult_batch.  Every k_p
 * must give the cone grids the operator was initialised with (else
 * IFGF_ERR_INVALID_ARG; a convolution-quadrature frequency set of the
 * modified Helmholtz kernel does); orders stay the operator's.  The planes
 * share the tree, cone maps and the geometry of one pass (node and source
 * positions, cone lookups, Chebyshev bases), each evaluating its own kernel
 * values and factors: one launch per stage and level for up to 64
 * wavenumbers (mixed precision, low orders (2,5,5), (3,6,6) or (4,7,7)).
 * FP64 runs ifgf_set_wavenumber and one matvec per wavenumber.  Replaces the
 * reference's operator-per-frequency loop (test/test_CQIFGF.cpp:117-135). */
int ifgf_mult_wavenumbers(ifgf_operator* op, const double* k, long n_k, const void* w, void* u);

/* ifgf_mult_wavenumbers on device buffers enqueued on `stream` (k stays a
 * host array).  No reference counterpart. */
int ifgf_mult_wavenumbers_device(ifgf_operator* op, const double* k, long n_k, const void* d_w,
                                 void* d_u, void* stream);

/* ifgf_mult on device buffers (complex128 / float64 as above) enqueued on
 * `stream` (a cudaStream_t, NULL = legacy default stream).  Returns after
 * enqueueing.  No reference counterpart. */
int ifgf_mult_device(ifgf_operator* op, const void* d_w, void* d_u, void* stream);

/* ifgf_mult_device for callers that cannot allocate device memory while they
 * apply the operator: an application whose own memory pool has reserved the
 * whole GPU (a cudaMalloc would fail or take memory the pool counts on), or
 * a real-time loop that must not stall on the implicit device
 * synchronisation of cudaMalloc / cudaFree.  This call allocates and frees
 * nothing: its per-call scratch lives in a fixed 64 MiB device array that the
 * library holds on every GPU that loads it, instead of the buffers init
 * allocated.  Operators whose matvec scratch exceeds 64 MiB are rejected with
 * IFGF_ERR_INVALID_ARG (use ifgf_mult_device for them); a current device
 * other than the one the operator was initialised on gives IFGF_ERR_STATE.
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  All calls share the one array and it
 * keeps the last call's contents, so calls whose GPU work overlaps (two
 * streams, two threads, two operators) race and must be serialised.  No
 * reference counterpart. */
int ifgf_mult_device_noalloc(ifgf_operator* op, const void* d_w, void* d_u, void* stream);

/* u = (dA/dk) w: the matvec of the wavenumber derivative of the kernel,
 * for the Helmholtz kernel (dG/dk = i e^{ikr}/(4 pi)) and the combined-field
 * kernel (e^{i kap r}/(4 pi r) (kap (n.(y - x) + r) - i)); other kernels
 * return IFGF_ERR_INVALID_ARG.  It runs on the operator's tree, cones and
 * orders with the derivative kernel factored by e^{ik r_c}/(4 pi); the first
 * call tabulates its upward geometry.  Buffers as in ifgf_mult_batch (host)
 * and ifgf_mult_device (device).  No reference counterpart: the reference
 * has no k-derivative; gradients with respect to k of a matvec are
 * (dA/dk) w. */
int ifgf_mult_dk(ifgf_operator* op, const void* w, void* u, long batch);
int ifgf_mult_dk_device(ifgf_operator* op, const void* d_w, void* d_u, void* stream);

/* u = A^H w, the adjoint matvec: w has one value per target, u one per
 * source (u_s = sum_t conj(G(x_s - y_t)) w_t).  Laplace, Helmholtz and
 * modified Helmholtz: conj(A' conj(w)) with A' the operator with sources and
 * targets exchanged (A itself when init got the same points twice); the
 * gradient kernel: minus that; double layer and combined field: composed
 * from three exchanged gradient operators (dG/dn_s = sum_d n_s[d] G_grad,d)
 * and, for the combined field, an exchanged Helmholtz operator.  The
 * operators are built on the first call from init's points, normals and
 * cutoff callback (which must therefore stay valid).  Buffers as in
 * ifgf_mult_batch / ifgf_mult_device with the roles of n_src and n_tgt
 * exchanged.  No reference counterpart: gradients of sum |A w - b|^2 with
 * respect to w are A^H (A w - b). */
int ifgf_mult_adjoint(ifgf_operator* op, const void* w, void* u, long batch);
int ifgf_mult_adjoint_device(ifgf_operator* op, const void* d_w, void* d_u, void* stream);

/* FP64 dense direct sum u(y_t) = sum_s w_s G(x_s - y_t) on the GPU at the
 * targets listed in tidx (caller's target indices), for error estimates:
 * w as in ifgf_mult (host buffer), out receives nt values.  The reference
 * checks its mult the same way on the host (test/test_ifgf.cpp:143-165). */
int ifgf_direct_eval(ifgf_operator* op, const void* w, const long* tidx, long nt, void* out);
/* ifgf_direct_eval of the k-derivative kernel (see ifgf_mult_dk).  No
 * reference counterpart. */
int ifgf_direct_eval_dk(ifgf_operator* op, const void* w, const long* tidx, long nt, void* out);

/* Per-kernel CUDA-event timing of every following mult (on the stream the
 * kernels run on); on != 0 enables and resets the counters.  Results appear
 * under "profile" in ifgf_stats_json.  No reference counterpart. */
int ifgf_set_profiling(ifgf_operator* op, int on);

int ifgf_num_sources(const ifgf_operator* op, long* n);
int ifgf_num_targets(const ifgf_operator* op, long* n);

/* Structured statistics of the last init/mult as JSON text (levels, boxes,
 * active cones, near/far pairs, per-stage milliseconds, work counts).
 * Writes at most cap bytes including the terminating NUL; *needed receives
 * the full length.  No reference counterpart (it prints to stdout). */
int ifgf_stats_json(const ifgf_operator* op, char* buf, long cap, long* needed);

/* Tree and cone tables, for parity tests against the reference's octree.
 * which: 0 = source tree, 1 = target tree.  ifgf_tree_levels and
 * ifgf_tree_num_boxes replace Octree::levels and Octree::numBoxes
 * (octree.hpp:884, :915). */
int ifgf_tree_levels(const ifgf_operator* op, int which, int* levels);
int ifgf_tree_num_boxes(const ifgf_operator* op, int which, int level, long* n);
/* perm[i] = original index of the i-th point in Morton order
 * (Octree::permutation, octree.hpp:225-226). */
int ifgf_tree_permutation(const ifgf_operator* op, int which, long* perm);
/* per box 12 longs: first, last, parent, is_leaf, child[8] (-1 = absent);
 * bbox: 6 doubles per box (min xyz, max xyz) (octree.hpp:1106-1184). */
int ifgf_tree_boxes(const ifgf_operator* op, int which, int level, long* ints, double* bbox);
/* interaction list of one source box (Octree::OctreeNode::nearTargets /
 * farTargets, octree.hpp:150-156): far = 0 near, 1 far; writes up to cap
 * (first, last) target point ranges in discovery order. */
int ifgf_box_list(const ifgf_operator* op, int level, long box, int far, long* out, long cap,
                  long* n);
/* active cone element ids of one source box, step 0 = fine, 1 = coarse,
 * in increasing element order (octree.hpp:743-790 hands them out in first-
 * insertion order; the set is the same). */
int ifgf_box_cones(const ifgf_operator* op, int level, long box, int step, long* out, long cap,
                   long* n);
/* cone grid of a level: n[3] elements per dimension (the level's
 * ConeDomain, octree.hpp:113, sized by elementsForBox,
 * ifgfoperator.hpp:99); orders of a step (orderForBox,
 * ifgfoperator.hpp:96) */
int ifgf_level_grid(const ifgf_operator* op, int level, int step, long* n);
int ifgf_orders(const ifgf_operator* op, int step, int* order);

/* Destroys the handle and frees its device memory (the operator's
 * destructor, ifgfoperator.hpp:61). */
int ifgf_destroy(ifgf_operator* op);

/* Message of the calling thread's last failed call ("" if none).  No
 * reference counterpart: the reference reports errors through assert and
 * C++ exceptions (pybind11 turns them into Python exceptions). */
const char* ifgf_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* IFGF_B200_H */
