/*
 * fmmb — a B200-native (sm_100a) fast multipole backend for FlexibleFMM.jl.
 *
 * C ABI. Every entry point returns a status code (FMMB_OK = 0) and leaves a message
 * for the calling thread in fmmb_last_error(). Handles are opaque; the caller owns its
 * arrays. Host-pointer entry points copy in and out and return when the results are in
 * host memory; `_dev` entry points take device pointers and only enqueue work on the
 * context's stream (synchronise with fmmb_ctx_synchronize or on the stream).
 *
 * Layouts follow the Julia memory of the reference types: points are D×N interleaved
 * (Vector{SVector{3,Float64}}), gradients 3×N interleaved (Vector{SVector{3,Float64}}),
 * node arrays are 0-based with -1 for "none". Inputs and outputs are in the caller's
 * original order; the tree order is internal (src/evaluate.jl:111-127 of the reference).
 *
 * Status codes map to the reference's exceptions: FMMB_ERR_ARGUMENT ↔ ArgumentError,
 * FMMB_ERR_DIMENSION ↔ DimensionMismatch.
 */
#ifndef FMMB_H
#define FMMB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FMMB_OK 0
#define FMMB_ERR_ARGUMENT 1    /* ArgumentError: non-finite points, outside the box, max_levels, bad option */
#define FMMB_ERR_DIMENSION 2   /* DimensionMismatch: lengths that do not match the plan */
#define FMMB_ERR_MEMORY 3      /* device or host allocation failed */
#define FMMB_ERR_DEVICE 4      /* a CUDA error */
#define FMMB_ERR_TIMEOUT 5     /* a bounded device wait gave up */
#define FMMB_ERR_UNSUPPORTED 6 /* a method, kernel, density or output the library does not provide */

#define FMMB_KERNEL_LAPLACE3D 1
#define FMMB_KERNEL_YUKAWA3D 2    /* e^{−κr}/(4πr), SphericalHarmonics(Yukawa3D(κ); p): FP64 path, operators per width */
#define FMMB_KERNEL_STOKESLET3D 3 /* StokesHarmonics(Stokeslet3D(); p): FP64 path; stokeslets, stresslets, doublets; velocity, pressure */
#define FMMB_KERNEL_LAPLACE2D 4   /* c·log r², c = −1/(4π): the circle KI method, points in the plane z = 0 */
#define FMMB_METHOD_SPHERICAL_HARMONICS 1
#define FMMB_METHOD_CUBE_KI 2 /* CubeKernelIndependent{3}(Laplace3D(); p, pc, d): spectral (FFT) M2L */
#define FMMB_METHOD_KI_CIRCLE 3 /* KernelIndependent(Laplace2D(); nequiv = p) (src/operators/kifmm.jl:17-33): 2D
                                   points given as 3×n with z = 0 (the binding embeds them), bbox origin
                                   z = −width/2; gradients come back with a zero z component */

#define FMMB_PRECISION_FP64 0  /* the plain path: FP64 everywhere (the drop-in) */
#define FMMB_PRECISION_MIXED 1 /* split-precision tensor-core M2L, FP32 compensated near field */

#define FMMB_OUTPUT_POTENTIAL 1 /* bit flags; both may be requested in one call */
#define FMMB_OUTPUT_GRADIENT 2

typedef struct fmmb_ctx fmmb_ctx;
typedef struct fmmb_cache fmmb_cache;
typedef struct fmmb_plan fmmb_plan;
typedef struct fmmb_state fmmb_state;

/* The method: SphericalHarmonics(Laplace3D(); p) (src/operators/harmonics.jl:303-308); with kernel
 * FMMB_KERNEL_YUKAWA3D SphericalHarmonics(Yukawa3D(kappa); p) (src/operators/harmonics_yukawa.jl:27-32);
 * with FMMB_KERNEL_STOKESLET3D StokesHarmonics(Stokeslet3D(); p) (src/operators/harmonics_stokes.jl:34-45);
 * with method FMMB_METHOD_CUBE_KI CubeKernelIndependent{3}(Laplace3D(); p, pc, d, pinv_rtol)
 * (src/operators/cubeki.jl:18-48). */
typedef struct {
  int32_t method;  /* FMMB_METHOD_SPHERICAL_HARMONICS or FMMB_METHOD_CUBE_KI */
  int32_t kernel;  /* FMMB_KERNEL_* (the cube KI method: FMMB_KERNEL_LAPLACE3D) */
  int32_t p;       /* harmonics: expansion degree, 1..20; cube KI: points per edge, 2..12; circle KI: nequiv, 4..64 */
  int32_t reserved;
  double tol;      /* 0: dense class operators (the only form the library provides) */
  double kappa;    /* the Yukawa screening κ > 0 (FMMB_KERNEL_YUKAWA3D); ignored otherwise */
  int32_t pc;      /* cube KI: points per edge of the large surface; 0: 2p */
  int32_t reserved2;
  double d;        /* cube KI: the surfaces' margin, in (0, 2/3); 0: 0.1 */
  double pinv_rtol; /* KI: the pseudo-inverses' truncation; 0: the reference's default, 50·eps(Float32) for
                       the cube method (Laplace3D(Float32)), 50·eps(Float64) for the circle method */
} fmmb_method_desc;

/* Tree options: FMM(m, sources; ppl, bbox, max_levels) (src/fmm.jl:31-49). */
typedef struct {
  int32_t ppl;        /* points per leaf; a node with more is split */
  int32_t max_levels; /* the reference default is 30 */
  int32_t has_bbox;   /* 0: the points' own square box (square_bbox) */
  int32_t reserved;
  double origin[3];   /* bbox = (origin, width) */
  double width;
} fmmb_tree_opts;

const char* fmmb_last_error(void);
const char* fmmb_version(void);

/* A device context: one GPU, one stream, the device-side scratch of the entry points. */
int fmmb_ctx_create(int device, fmmb_ctx** out);
int fmmb_ctx_destroy(fmmb_ctx* ctx);
int fmmb_ctx_stream(fmmb_ctx* ctx, void** stream); /* the cudaStream_t all work goes to */
int fmmb_ctx_synchronize(fmmb_ctx* ctx);

/* OperatorCache(method) (src/operators/cache.jl:19-22): operators by box width, their device
 * copies shared by every plan built with the cache. The first plan fixes the base width. */
int fmmb_cache_create(fmmb_ctx* ctx, const fmmb_method_desc* method, fmmb_cache** out);
int fmmb_cache_destroy(fmmb_cache* cache);
int fmmb_cache_base_width(const fmmb_cache* cache, double* width); /* NaN until a box was fitted */

/* FMM(method, sources; ppl, bbox, cache, max_levels) (src/fmm.jl:31-49) and
 * DevicePlan(m, xs; ...) (src/device_passes.jl:112-134): the tree of the points, built on
 * the device, the box snapped by fit_box! (src/operators/cache.jl:57-83), the interaction
 * lists and the operators of every level. xyz: 3×n interleaved. */
int fmmb_plan_create(fmmb_cache* cache, const double* xyz, int64_t n, const fmmb_tree_opts* opts, fmmb_plan** out);
int fmmb_plan_create_dev(fmmb_cache* cache, const double* xyz_dev, int64_t n, const fmmb_tree_opts* opts, fmmb_plan** out);
int fmmb_plan_destroy(fmmb_plan* plan);
/* info[0] = levels, info[1] = nodes, info[2] = points, info[3] = far pairs,
 * info[4 .. 4+levels] = first node of each level and the node count, then (if cap allows) the
 * targets per M2L block (cap: entries of info, at least 5 + levels). */
int fmmb_plan_info(const fmmb_plan* plan, int64_t* info, int cap);
int fmmb_plan_box(const fmmb_plan* plan, double* origin3, double* width);
/* The flat tree (src/tree/tree.jl:40-71), downloaded: any pointer may be NULL.
 * cell 3×nnodes, level (0 = root), parent, child_first, plo/phi (0-based inclusive point
 * range, phi < plo when empty), flags (bit 0 leaf, 1 ghost, 2 xlist, 3 has_source),
 * colleagues 27×nnodes, perm (sorted position → original index), point_node. */
int fmmb_plan_tree(const fmmb_plan* plan, int32_t* cell, int32_t* level, int32_t* parent, int32_t* child_first,
                   int32_t* plo, int32_t* phi, uint8_t* flags, int32_t* colleagues, int32_t* perm, int32_t* point_node);
/* The far pairs of one level as (target node, source node, far offset index) in an
 * unspecified order (src/tree/lists.jl:15-70); returns the count in *npairs. */
int fmmb_plan_pairs(const fmmb_plan* plan, int level, int32_t* tgt, int32_t* src, int32_t* far, int64_t cap, int64_t* npairs);

/* A batch of independent FMMs in one plan (no counterpart in the reference, whose DevicePlan(m,
 * groups) puts several point sets in ONE tree, src/device_passes.jl:112-134): ninst point sets,
 * instance i the counts[i] points after those of instances 0..i-1 in xyz (3 × Σcounts), each with
 * its own tree in its own box (boxes: 4 per instance, origin and width; NULL: each set's
 * square_bbox), the boxes fitted by fit_box! in instance order exactly as plans created one after
 * another with this cache would be. One tree build, one list build, and one launch per pass and
 * level serve every instance; each instance's tree, far pairs and results are bitwise those of its
 * own plan (fmmb_plan_create with the same cache, box and options). The states, builds and
 * evaluations at the sources take the plan like any other, with all instances' points, densities
 * and outputs concatenated in instance order; evaluations at targets are not provided for a batch
 * (FMMB_ERR_UNSUPPORTED), nor the kernel-independent methods. Levels are global: level l holds the
 * nodes of width ldexp(W, -l), W the widest root's, and an instance's root lies on the level of its
 * width. */
int fmmb_batch_plan_create(fmmb_cache* cache, const double* xyz, const int64_t* counts, int64_t ninst,
                           const fmmb_tree_opts* opts, const double* boxes, fmmb_plan** out);
int fmmb_batch_plan_create_dev(fmmb_cache* cache, const double* xyz_dev, const int64_t* counts, int64_t ninst,
                               const fmmb_tree_opts* opts, const double* boxes, fmmb_plan** out);
/* The instances of a plan (1 for a plan of one point set): *ninst, and where not NULL offsets
 * (ninst + 1: the first point of each instance, then the total), boxes (4 × ninst), root_level
 * (ninst: the global level of each root) and node_instance (nnodes). */
int fmmb_batch_plan_instances(const fmmb_plan* plan, int64_t* ninst, int64_t* offsets, double* boxes,
                              int32_t* root_level, int32_t* node_instance);

/* The autotuner (no counterpart in the reference): times the launch shapes of a state's matvec on
 * the given inputs (the plan's points, n of them, and its charges, or 3×n Stokeslets) — the M2L
 * block size (32, 64, 128 targets; when tune_blocks, re-cutting the plan's blocks, which its other
 * states share), the FP64 M2L's chunk width, the near field's warps per CTA — keeps the fastest
 * and applies it, and records it for later plans and states of the same method, kernel, order,
 * precision path and N rounded down to a power of two. No result depends on these shapes. The
 * state's expansions must be built again afterwards. out (may be NULL): 5 doubles, the block
 * size, the chunk-width variant, the warps, and the chosen M2L and near-field times in ms. */
int fmmb_autotune(fmmb_state* state, const double* xyz, const double* tau, int64_t n, int tune_blocks, double* out);
int fmmb_autotune_dev(fmmb_state* state, const double* xyz_dev, const double* tau_dev, int64_t n, int tune_blocks,
                      double* out);

/* FMMState (src/fmm.jl:64-94): the expansions of one right-hand side, in a precision path. */
int fmmb_state_create(fmmb_plan* plan, int precision, fmmb_state** out);
int fmmb_state_destroy(fmmb_state* state);

/* build_expansions!(state, fmm, sources, τ) (src/fmm.jl:270-298) with charges τ. */
int fmmb_build_expansions(fmmb_state* state, const double* xyz, const double* tau, int64_t n);
int fmmb_build_expansions_dev(fmmb_state* state, const double* xyz_dev, const double* tau_dev, int64_t n);
/* build_expansions! with Dipole densities, alone or with charges (τ as a tuple of a charge and a
 * Dipole per source, src/sources.jl:16-31, src/operators/harmonics.jl:708-738): tau n charges or
 * NULL, dipoles 3×n moments d (field d·∇ₛG) or NULL; SphericalHarmonics(Laplace3D) on either
 * precision path. The evaluation of a state built this way takes the dipoles' near field. */
int fmmb_build_expansions_dipoles(fmmb_state* state, const double* xyz, const double* tau, const double* dipoles, int64_t n);
int fmmb_build_expansions_dipoles_dev(fmmb_state* state, const double* xyz_dev, const double* tau_dev,
                                      const double* dipoles_dev, int64_t n);
/* evaluate_at_sources!(out, fmm, state; output) (src/evaluate.jl:111-127): pot (n) and/or
 * grad (3×n) in the original order, self excluded. */
int fmmb_evaluate_at_sources(fmmb_state* state, int outputs, double* pot, double* grad);
int fmmb_evaluate_at_sources_dev(fmmb_state* state, int outputs, double* pot_dev, double* grad_dev);
/* device_matvec! (src/device_passes.jl:619-640): build_expansions then evaluate_at_sources. */
int fmmb_matvec(fmmb_state* state, const double* xyz, const double* tau, int64_t n, int outputs, double* pot, double* grad);
int fmmb_matvec_dev(fmmb_state* state, const double* xyz_dev, const double* tau_dev, int64_t n, int outputs,
                    double* pot_dev, double* grad_dev);
/* evaluate!(out, fmm, state, targets; output) (src/evaluate.jl:81-96): targets 3×nt, located
 * on the device (src/tree/locate.jl:10-22). */
int fmmb_evaluate(fmmb_state* state, const double* targets, int64_t nt, int outputs, double* pot, double* grad);
int fmmb_evaluate_dev(fmmb_state* state, const double* targets_dev, int64_t nt, int outputs, double* pot_dev, double* grad_dev);
/* Waits for the state's work on the context's stream and reports what its kernels flagged:
 * FMMB_ERR_TIMEOUT when a bounded wait of the tensor-core M2L gave up since the last report
 * (the expansions of that build are incomplete). The host-pointer entry points report it
 * themselves; callers of the _dev entry points call this where they synchronise. No
 * counterpart in the reference (its calls are synchronous). */
int fmmb_state_synchronize(fmmb_state* state);
/* One device matvec (fmmb_matvec_dev) with CUDA events between its stages, on the context's
 * stream, synchronised: stage_ms[0..5] = gather, P2M, M2M, M2L (with the zeroing of the partial
 * locals and, on the mixed path, the FP32 copy of the multipoles), L2L, evaluation (L2P + P2P).
 * *launches = the kernels launched (the reference times the same phases: bench/bench.jl:44-56). */
int fmmb_profile_matvec(fmmb_state* state, const double* xyz_dev, const double* tau_dev, int64_t n, int outputs,
                        double* pot_dev, double* grad_dev, double* stage_ms, int cap, int* launches);
/* The multipoles and locals of the last build (nnodes × nexp × (p+1)² each, node order, the real
 * storage of src/operators/harmonics.jl:20-27, nexp = 1 for Laplace3D and 4 (Φ₁, Φ₂, Φ₃, Ψ̂) for
 * the Stokeslet; locals are zero outside the real leaves). */
int fmmb_state_expansions(const fmmb_state* state, double* multipoles, double* locals);

/* stokes_fmm_eval!(velocities, plan; stokeslets) with a self plan (src/stokes_api.jl:131-150) on a
 * state of a Stokeslet cache (FP64 path): build_expansions! then evaluate_at_sources!, the i = j
 * term skipped. xyz 3×n, stokeslets 3×n (Vector{SVector{3,Float64}}), velocity 3×n out, all in
 * the original order. The Laplace entry points reject Stokeslet states (FMMB_ERR_UNSUPPORTED). */
int fmmb_stokes_eval(fmmb_state* state, const double* xyz, const double* stokeslets, int64_t n, double* velocity);
int fmmb_stokes_eval_dev(fmmb_state* state, const double* xyz_dev, const double* stokeslets_dev, int64_t n,
                         double* velocity_dev);

/* The densities of stokes_fmm_eval! (src/stokes_api.jl:72-83,107-123): any of stokeslets,
 * stresslets with stressvecs (both or neither), doublets, each 3×n in the original order or NULL,
 * at least one given; weights (n or NULL) multiply the stokeslets, the stresslet strengths and the
 * doublets. Fields (src/sources.jl:203-281, c = 1/8π, d = t − s): stokeslet c(f/r + d(d·f)/r³),
 * Stresslet(f, ν) −6c d(d·f)(d·ν)/r⁵, Doublet(g) c(g/r³ − 3d(d·g)/r⁵); pressures 2c(d·f)/r³,
 * 4c[(f·ν)/r³ − 3(d·f)(d·ν)/r⁵] and 0. */
typedef struct fmmb_stokes_densities {
  const double* stokeslets;
  const double* stresslets;
  const double* stressvecs;
  const double* doublets;
  const double* weights;
} fmmb_stokes_densities;

#define FMMB_STOKES_VELOCITY 0 /* Velocity(): 3×n out */
#define FMMB_STOKES_PRESSURE 1 /* Pressure(): n out */
#define FMMB_STOKES_GRADIENT 2 /* Gradient(): 9×n out, ∂u_i/∂t_j at 9·k + 3·i + j (row-major per point) */

/* stokes_fmm_eval!(out, plan; stokeslets, stresslets, stressvecs, doublets, weights, output) with
 * a self plan (src/stokes_api.jl:107-123) on a Stokeslet state: the velocities or pressures at the
 * sources, the i = j term skipped. Host pointers (the densities' pointers too); the _dev form
 * takes device pointers for xyz, every density array and out (dens itself is a host struct).
 * ArgumentError for no density or a stresslet without its stressvecs. */
int fmmb_stokes_eval_densities(fmmb_state* state, const double* xyz, const fmmb_stokes_densities* dens, int64_t n,
                               int output, double* out);
int fmmb_stokes_eval_densities_dev(fmmb_state* state, const double* xyz_dev, const fmmb_stokes_densities* dens,
                                   int64_t n, int output, double* out_dev);

/* stokes_fmm_eval! with a plan that has targets, and stokes_fmm_eval_src_trg! (src/stokes_api.jl:
 * 107-146): one build_expansions!, then the outputs at the sources (out_src, i = j skipped; NULL to
 * skip) and at nt targets (3×nt, inside the plan's box, else ArgumentError; out_trg, NULL to
 * skip), velocities 3 per point or pressures 1 per point, in the original orders. */
int fmmb_stokes_eval_src_trg(fmmb_state* state, const double* xyz, const fmmb_stokes_densities* dens, int64_t n,
                             const double* targets, int64_t nt, int output, double* out_src, double* out_trg);
int fmmb_stokes_eval_src_trg_dev(fmmb_state* state, const double* xyz_dev, const fmmb_stokes_densities* dens,
                                 int64_t n, const double* targets_dev, int64_t nt, int output, double* out_src_dev,
                                 double* out_trg_dev);

/* direct!(out, K, sources, τ, targets) / direct_self! (src/kernels.jl:463-487) for Laplace3D on
 * the device in FP64, device pointers: sources 3×ns, targets 3×nt. self_index (device, may be
 * NULL): per target, the source index it excludes (-1 for none). */
int fmmb_direct_dev(fmmb_ctx* ctx, const double* src_dev, const double* tau_dev, int64_t ns, const double* tgt_dev,
                    const int64_t* self_index_dev, int64_t nt, double* pot_dev, double* grad_dev);

/* fmmb_direct_dev without any device allocation, for callers that cannot call cudaMalloc: an
 * application whose device memory is held by its own pool (CUDA.jl's allocator keeps what it
 * reserved) or a time-stepping loop that must not pay cudaMalloc's implicit synchronisation.
 * No counterpart in the reference. Same arguments and results as fmmb_direct_dev; enqueues on
 * the context's stream and returns without synchronising. The partial sums live in a 4 MiB
 * array compiled into the library (held by every GPU that loads it until exit), so nt is
 * limited to 131,072 targets (FMMB_ERR_ARGUMENT above). All calls share that array: calls that
 * overlap on the GPU race. The array's device address is looked up when the context is created
 * (fmmb_ctx_create), which loads the library's device code then rather than inside a call, and
 * again in a new CUDA context (after a device reset); create the context before any stream
 * capture. */
int fmmb_direct_noalloc_dev(fmmb_ctx* ctx, const double* src_dev, const double* tau_dev, int64_t ns,
                            const double* tgt_dev, const int64_t* self_index_dev, int64_t nt, double* pot_dev,
                            double* grad_dev);

/* A continuous-batching request server on one GPU (no counterpart in the reference, which runs
 * one FMM per call: this is the serving form of FMM + build_expansions + evaluate_at_sources).
 * Requests are admitted in arrival order onto `slots` worker threads, each with its own context
 * (stream) and an operator cache per order that stays resident, as soon as a slot is free and
 * the request's estimated device memory fits what the requests in flight leave of hbm_budget
 * (the front request waits rather than being overtaken; one that exceeds the budget alone runs
 * when nothing else does). The device work of admitted requests overlaps. A slot takes the front
 * request together with later queued requests of the same kind (kernel, order, precision path,
 * κ, ppl, outputs), up to group_max requests and group_points points that fit the budget, and
 * runs them as one batch plan (fmmb_batch_plan_create): one tree build, one list build and one
 * launch per pass for the group. Each request is computed exactly as it would be alone (its
 * results are bitwise the same in any mix and any group). */
typedef struct fmmb_server fmmb_server;
typedef struct {
  int32_t slots;       /* concurrent groups (worker threads, one stream each), 1..64 */
  int32_t ppl;         /* points per leaf of every request's tree; 0: by the request's order and path
                          (64 on the mixed path and up to p = 8, 128 to p = 13, 256 to 17, 512 above) */
  int64_t hbm_budget;  /* bytes of device memory the admitted requests may hold; 0: 80 % of the free memory */
  int32_t group_max;   /* requests per group; 0: 64; 1: every request alone */
  int32_t reserved;
  int64_t group_points; /* points per group (a larger request runs alone); 0: 4,000,000 */
} fmmb_server_opts;
typedef struct {
  const double* xyz;   /* 3×n host, original order; read while the request runs */
  const double* tau;   /* n host charges (Laplace3D); 3×n Stokeslets (Stokeslet3D) */
  int64_t n;
  double tol;          /* requested relative accuracy: selects p (when p = 0) and the precision path */
  int32_t kernel;      /* FMMB_KERNEL_LAPLACE3D, FMMB_KERNEL_YUKAWA3D (FP64), or FMMB_KERNEL_STOKESLET3D
                          (velocities at the sources) */
  int32_t p;           /* 0: the smallest order whose measured error is below tol */
  int32_t outputs;     /* FMMB_OUTPUT_* bits (Laplace3D) */
  int32_t precision;   /* -1: FP64 for tol < 1e-8 or p > 11, else the mixed path (Stokeslet3D: FP64) */
  int32_t ppl;         /* points per leaf of this request's tree; 0: the server's */
  double* pot;         /* n host potentials, or 3×n velocities; written when the request completes
                          (keep valid until then) */
  double* grad;        /* 3×n host */
  double kappa;        /* the Yukawa screening κ (FMMB_KERNEL_YUKAWA3D) */
} fmmb_request;
typedef struct {
  int32_t status;      /* the request's own status (FMMB_OK or an error code) */
  int32_t p, precision, slot;
  double queued_s;     /* submission → admission */
  double run_s;        /* admission → results in host memory */
  double latency_s;    /* submission → results in host memory */
  int64_t bytes_estimate;
  double plan_s;       /* host time of the plan (tree, lists, operators) and the state */
  double matvec_s;     /* host time of the matvec (copies in, kernels, copies out) */
  double device_s;     /* the matvec's span on the slot's stream (CUDA events around it) */
  int32_t group;       /* requests in this request's group; the three times above are the group's
                          divided by it (so that they sum to the group's over its requests) */
  int32_t reserved;
} fmmb_request_info;
int fmmb_server_create(int device, const fmmb_server_opts* opts, fmmb_server** out);
int fmmb_server_submit(fmmb_server* server, const fmmb_request* request, int64_t* ticket);
/* Wait for a request (timeout_s < 0: without limit; FMMB_ERR_TIMEOUT if it is not done in time,
 * the ticket stays valid); returns the request's status. A ticket is waited for once. */
int fmmb_server_wait(fmmb_server* server, int64_t ticket, double timeout_s, fmmb_request_info* info);
/* Stops accepting requests, finishes the queued and running ones, then releases everything. */
int fmmb_server_destroy(fmmb_server* server);

/* Test hook of the bounded waits (no counterpart in the reference): until called again with
 * slab = -1, the tensor-core M2L launches stop reporting K-step slab number `slab` of every
 * block as gathered and give each wait `wait_seconds` (default one second when ≤ 0), so that
 * the waits run out, every role gives up, the kernel frees its tensor memory and returns, and
 * the next synchronising call reports FMMB_ERR_TIMEOUT. Process-wide; for tests only. */
int fmmb_test_m2l_stall(int64_t slab, double wait_seconds);

#ifdef __cplusplus
}
#endif

#endif /* FMMB_H */
