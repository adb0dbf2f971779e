// The context, operator cache, plan (tree + lists) and state (expansions) of the library.
#pragma once
#include <map>
#include <memory>
#include <mutex>

#include "common.cuh"
#include "ki.h"

namespace fmmb {

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
};

// The Yukawa operators of one box width (src/operators/harmonics_yukawa.jl:164-207): the 34
// class representatives with c_K / w folded in, M2M (children of width w/2 into the parent) and
// L2L (the parent into its children), in the Laplace layouts.
struct YukawaLevel {
  DBuf<double> reps, m2m, l2l;
  // the mixed path's split class operators of this width (built when a mixed state first needs
  // them, like the cache's reps16/row_scale for the homogeneous kernels)
  std::mutex mu;
  DBuf<uint16_t> reps16;
  DBuf<float> row_scale;
};

// OperatorCache (src/operators/cache.jl:5-83): the base width, the host operators at the base
// width and their device copies, shared by every plan built with the cache.
struct Cache {
  Ctx* ctx = nullptr;
  int p = 0, np = 0, ld = 0;
  int kernel = FMMB_KERNEL_LAPLACE3D;
  int nexp = 1;              // scalar expansions per node: 1 (Laplace3D), 4 (Stokeslet3D: Φ₁..₃, Ψ̂)
  double W0 = NAN;           // base width, fixed by the first fitted box
  std::mutex mu;             // the cache is shared by plans; fitting and uploads are locked
  bool uploaded = false;
  HostOperators host;
  DBuf<double> m2m, l2l, reps, tables;
  DBuf<int16_t> gidx, sidx;
  DBuf<int8_t> gsgn, ssgn;
  DBuf<int> cls;
  // the mixed path's class operators (m2l_tc.cu): per class, the row-scaled FP16 head and
  // tail in the canonical K-major layout of the tensor-core M2L; the inverse row scales; the
  // source-side sign words and byte selectors of the D4h permutations
  DBuf<uint16_t> reps16;
  DBuf<float> row_scale;
  DBuf<uint32_t> perm16;
  bool split_ready = false;
  // Yukawa3D: κ, the operators per width (keyed by the exponent e of w = ldexp(W0, e); built on
  // first use and shared by every cache of the same device, order, κ and width), and the sphere
  // quadrature of the projections
  double kappa = 0;
  std::map<int, std::shared_ptr<YukawaLevel>> yk_levels;
  DBuf<double> yk_xq, yk_wq;
  int yk_nq = 0;
  // CubeKernelIndependent{3}: the method, its parameters, the host operators at width 1 (shared
  // by caches with the same parameters) and their device copies at width 1 (surfaces, factored
  // pseudo-inverses padded to RU/RD/NLD rows, M2M/L2L in the Laplace layouts, spectral tables
  // as float2 over nfp = nfreq rounded up to 64 frequencies)
  int method = FMMB_METHOD_SPHERICAL_HARMONICS;
  int ki_pc = 0;
  double ki_d = 0, ki_rtol = 0;
  std::shared_ptr<const KIHost> ki;
  int ki_nl = 0, ki_nld = 0, ki_ru = 0, ki_rd = 0, ki_nfp = 0;
  DBuf<double> ki_large, ki_upv, ki_upsu, ki_downv, ki_downsu, ki_m2m, ki_l2l;
  DBuf<int> ki_embed;
  DBuf<float2> ki_tab, ki_tw;
  // KernelIndependent(Laplace2D()): circle operators per width (keyed by the exponent e of
  // w = ldexp(W0, e)), built on the host when a plan first needs that width
  struct CircleLevel { DBuf<double> upv, upsu, downv, downsu, m2m, l2l, m2l; };
  std::map<int, std::unique_ptr<CircleLevel>> kic_levels;
};

// One M2L work block: TB consecutive nodes of one segment (the targets), their far pairs
// grouped by symmetry class. On the device the level and the segment share one word
// (level | segment << 8).
struct M2LBlock {
  int level;
  int seg;
  int first;     // first node (global)
  int count;     // nodes in the block
  int pair_base; // first pair of the block in the plan's pair array
};

struct Plan {
  Cache* cache = nullptr;
  Ctx* ctx = nullptr;
  int64_t N = 0;
  int L = 0, nnodes = 0, KL = 21;
  double origin[3] = {0, 0, 0}, W0 = 1;
  int e0 = 0;                             // the plan's root width is ldexp(cache W0, e0)
  std::vector<int> level_start;           // L + 1
  std::vector<double> scale, m2l_scale;   // per level: 1/w, and the M2L factor W_ref / w
  // the flat tree on the device
  DBuf<int4> cell;                        // x, y, z, level
  DBuf<int> parent, cf, plo, phi, col, perm, point_node;
  DBuf<uint8_t> flags;
  // host copies of the node arrays the host-side scheduling needs
  std::vector<int> h_parent, h_cf, h_plo, h_phi;
  std::vector<uint8_t> h_flags;
  // upward: childless nodes with sources (all levels); per level the sibling-group parents
  DBuf<int> s2m_nodes;
  int n_s2m = 0;
  std::vector<DBuf<int>> group_parent;    // per level l ≥ 1: parent of each sibling group
  // evaluation: real leaves with points
  DBuf<int> leaves, leaf_start, leaf_count;
  int n_leaves = 0;
  // M2L: blocks, per block the class offsets of its pairs, the pairs (src, f << 8 | target)
  int TB = 128;
  std::vector<M2LBlock> h_blocks;
  DBuf<int4> blocks;
  DBuf<int> cls_off;                      // nblocks × 35, relative to the block's pair_base
  DBuf<int2> pairs;
  DBuf<int> rtab;                         // nblocks × 34 × TB: per class and target, count << 16 | offset in the class
  DBuf<int> rounds;                       // nblocks × 34: per class the largest count of a target
  int64_t npairs = 0;
  std::vector<int64_t> level_pairs;       // far pairs per level
  std::vector<int> h_pair_count;          // far pairs per target node (the blocks are cut from it)
  DBuf<double> d_scale, d_m2l_scale;      // per level
  // the translation operators of each level (the cache's for the homogeneous kernels; the
  // level's own width for Yukawa3D): M2L representatives, M2M into and L2L out of the level's
  // nodes; the representatives' table on the device for the M2L kernel; Yukawa3D's κ̂² per level
  std::vector<const double*> lv_reps, lv_m2m, lv_l2l;
  DBuf<uint64_t> d_lv_reps;
  DBuf<double> d_kh2;
  // the mixed path: per level the split class operators and their inverse row scales (the cache's
  // for the homogeneous kernels, the level width's own for Yukawa3D), built with the first mixed
  // state; the Yukawa levels they come from stay held by the plan
  DBuf<uint64_t> d_lv_reps16, d_lv_rsc;
  std::vector<std::shared_ptr<YukawaLevel>> lv_yukawa;
  // the kernel-independent method: every target's far pairs (source, far index), target-major
  DBuf<int> tp_ptr;
  DBuf<int2> tp;
  DBuf<int> ki_leaves;                    // every real leaf (with sources or not)
  int n_ki_leaves = 0;
  // the circle method: per level its pseudo-inverse factors, and the level ranges of the
  // childless nodes with sources and of the real leaves (both lists are in node order)
  std::vector<const double*> kic_upv, kic_upsu, kic_downv, kic_downsu;
  std::vector<int> s2m_level_start, ki_leaf_level_start;
  // per level its sibling groups: the level's first 8·level_groups[l] nodes (a batch's roots
  // below level 0 follow them)
  std::vector<int> level_groups;
  // a batch (several independent point sets in one forest): instance i is the input points
  // [inst_off[i], inst_off[i + 1]), its root box inst_box[4i..4i+3] (origin, width
  // ldexp(cache W0, inst_e[i])), its root on level inst_root[i]; per node its instance; the
  // segments (one instance's nodes of one level, contiguous): per node its segment (the mixed
  // path's scale index; a plan of one point set has one segment per level and no array)
  int ninst = 1;
  std::vector<int64_t> inst_off;
  std::vector<double> inst_box;
  std::vector<int> inst_e, inst_root;
  DBuf<int64_t> d_inst_off;
  DBuf<double> d_inst_box;
  DBuf<int> node_inst;
  std::vector<int> h_inst;
  std::vector<int> seg_start, seg_level, seg_inst;   // nseg (+ 1 for seg_start)
  DBuf<int> node_seg;
  int nseg = 0;
};

struct State {
  Plan* plan = nullptr;
  int precision = FMMB_PRECISION_FP64;
  // launch shapes chosen by the tuner (tune.cu): near-field warps per CTA (4 or 8), the FP64
  // M2L's alternative chunk width
  int near_warps = 4;
  int f64_nb_alt = 0;
  DBuf<double> xs, ys, zs, q;             // sources and charges in tree order
  DBuf<double> f3;                        // Stokeslet states: the forces in tree order (fx, fy, fz)
  DBuf<double> sd;                        //   stresslet strengths, stressvecs, doublets (3 × N planar each)
  DBuf<double> dip4;                      //   the four blocks' dipole densities (3 × N planar each)
  bool stokes_dens = false;               //   the last build had stresslets or doublets
  DBuf<double> dip;                       // dipole densities in tree order (dx, dy, dz: 3 × N planar)
  bool has_dip = false;                   // the last build had dipoles (the P2M and near field take them)
  DBuf<double> M, Pl;                     // nnodes × LD: multipoles, partial locals
  DBuf<uint16_t> Mh, Ml;                  // the mixed path: the multipoles scaled by a power of two
  DBuf<float> Lsc;                        //   per level, as FP16 head and tail; the inverse scales
  DBuf<unsigned long long> Lmax;          //   and the levels' largest entries
  DBuf<int> err;                          // the mixed path: the bounded-wait error flag
  // the kernel-independent method: check potentials of the childless nodes on their large
  // surfaces, the pseudo-inverses' middle products, the leaves' local densities on their large
  // surfaces (nnodes × NLD), the spectra of the multipoles and of the M2L sums (nnodes × nfp)
  DBuf<double> ki_pm, ki_y, ki_ll;
  DBuf<float2> ki_spec, ki_u;
  bool built = false;
  // the side stream of the split matvec (the near field beside the passes) and its two events,
  // created on first use
  struct Side {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    void ensure();
    ~Side();
  } side;
  // the side stream's work reads the state's buffers and writes the outputs: it ends before any
  // member is freed (an exception between the fork and the join leaves it unjoined)
  ~State() {
    if (side.s) cudaStreamSynchronize(side.s);
  }
  // staging of the host-pointer entry points and the evaluation at targets
  DBuf<double> h_in_xyz, h_in_tau, d_pot, d_grad;
  DBuf<double> t_x, t_y, t_z;
  DBuf<int> t_node, t_groups, t_out;
  DBuf<uint64_t> t_keys;
  DBuf<uint32_t> t_vals;
};

// tree.cu
void build_tree(Plan& P, const double* xyz_dev, int ppl, int max_levels);
// lists.cu
void build_lists(Plan& P);
void build_blocks(Plan& P, int TB);       // the M2L blocks of TB targets (re)cut from P.h_pair_count
// tune.cu: the tuned launch shapes of plans and states of a kind (method, kernel, p, precision,
// N rounded down to a power of two); 0 / unchanged where none was tuned
int tuned_block_size(const Plan& P);
void apply_tuned_state(State& S);
// times the launch shapes on the state's inputs, keeps the fastest for its kind and applies them
// (tune_blocks: also the plan's M2L block size, shared by the plan's other states); out: the
// chosen block size, FP64 chunk width variant, near-field warps, and the M2L and near-field ms
void autotune(State& S, const double* xyz_dev, const double* tau_dev, bool tune_blocks, double* out);
void build_target_pairs(Plan& P);
// passes.cu
void upload_operators(Cache& C);
void gather_inputs(State& S, const double* xyz_dev, const double* tau_dev);
// charges (tau, or none) and dipole moments (3 × n interleaved, or none) in original order
void gather_inputs_dipoles(State& S, const double* xyz_dev, const double* tau_dev, const double* dip_dev);
void upward_pass(State& S);
void downward_pass(State& S);
void evaluate_sources(State& S, int outputs, double* pot_dev, double* grad_dev);
void evaluate_targets(State& S, const double* tg_dev, int64_t nt, int outputs, double* pot_dev, double* grad_dev);
// locate nt > 0 targets (device, 3 × nt) in the tree's leaves (FMMB_ERR_ARGUMENT outside the box)
// and group them per leaf: S.t_x/t_y/t_z in leaf order, S.t_out their original indices, and the ng
// groups (returned) as S.t_groups = [node; first; count] (ng each)
int group_targets(State& S, const double* tg_dev, int64_t nt);
// eval.cu: the evaluation at the sources split in two (harmonic methods with charges): the near
// field on stream st writes the outputs, the far field (on the state's stream, after it) adds
bool split_evaluation(const State& S);
void near_sources(State& S, int outputs, double* pot_dev, double* grad_dev, cudaStream_t st);
void far_sources(State& S, int outputs, double* pot_dev, double* grad_dev);
void bounds(Ctx& ctx, const double* xyz_dev, int64_t n, double lo[3], double hi[3], int64_t* nonfinite);
// the bounds of each instance of a batch (points [off[i], off[i + 1]) of xyz_dev): lo, hi 3 × ninst
void bounds_batch(Ctx& ctx, const double* xyz_dev, const std::vector<int64_t>& off, std::vector<double>& lo,
                  std::vector<double>& hi, int64_t* nonfinite);
void direct(Ctx& ctx, const double* src, const double* tau, int64_t ns, const double* tgt, const int64_t* self_idx,
            int64_t nt, double* pot, double* grad);
// ki.cu: CubeKernelIndependent{3}(Laplace3D()): cache and plan setup, the passes
void ki_prepare(Plan& P);
void ki_state(State& S);
int ki_p2m(State& S);
int ki_m2l(State& S);
int ki_leaf_locals(State& S);
// kic.cu: KernelIndependent(Laplace2D()) on circles, the points in the plane z = 0 of the octree
void kic_prepare(Plan& P);
void kic_state(State& S);
int kic_p2m(State& S);
int kic_m2l(State& S);
int kic_leaf_locals(State& S);
// yukawa.cu: SphericalHarmonics(Yukawa3D(κ)) — the operators of the plan's widths (built on the
// device by projection when a width is first used) and the per-level factors
void yukawa_prepare(Plan& P);
// stokes.cu: StokesHarmonics(Stokeslet3D()) on the FP64 path
// the densities of stokes_fmm_eval! (device, original order; each may be null, stresslets and
// stressvecs together): 3 × n each, weights n
struct StokesDensities {
  const double *stokeslets = nullptr, *stresslets = nullptr, *stressvecs = nullptr, *doublets = nullptr,
               *weights = nullptr;
};
void stokes_build(State& S, const double* xyz_dev, const StokesDensities& d);
// output FMMB_STOKES_VELOCITY (3 × n), FMMB_STOKES_PRESSURE (n) or FMMB_STOKES_GRADIENT (9 × n),
// original order, device
void stokes_evaluate_sources(State& S, int output, double* out_dev);
// the same at nt targets (device, 3 × nt) inside the tree's box, in the targets' order
void stokes_evaluate_targets(State& S, const double* tg_dev, int64_t nt, int output, double* out_dev);
// direct_noalloc.cu: the same sums with the partials in a fixed array compiled into the library
void direct_noalloc(Ctx& ctx, const double* src, const double* tau, int64_t ns, const double* tgt, const int64_t* self_idx,
                    int64_t nt, double* pot, double* grad);

}  // namespace fmmb
