// C ABI of the B200 MPS engine (include/vqemps.h): circuit compilation, the
// shared-prefix plan of a Pauli sum, workspaces and kernel launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <array>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/vqemps.h"
#include "common.cuh"
#include "evolve.cuh"
#include "expect.cuh"
#include "expect_mma.cuh"
#include "expect_real.cuh"
#include "sample.cuh"
#include "gradient.cuh"
#include "gradient_mma.cuh"

using namespace vqemps;

namespace {

struct Hamiltonian {
  int n = 0, T = 0;
  int nleaf = 0;
  int identity_leaf = -1;
  bool all_diagonal = true;
  std::vector<int32_t> term_leaf;        // T
  std::vector<double> leaf_coef;         // nleaf
  std::vector<int> group_off, node_off;  // n + 1 offsets into the flat arrays
  std::vector<int> nslot;                // env slots per level
  std::vector<DevGroup> groups;
  std::vector<DevNode> nodes;
  std::vector<int32_t> leaf_level;       // level of every leaf (-1: identity)
  int max_slot = 1;
  std::map<int, int> tuned;              // batch-size bucket -> level kernel variant
  // work accounting (FP64 real flops of one evaluation of one state)
  double flops = 0.0;
  double flops_survey = 0.0;
  long long node_sites = 0;
  // sampling support: Z masks over sites (one uint64 row per word), X/Y flags
  std::vector<uint64_t> zmask;           // T x W
  std::vector<uint8_t> offdiag;          // T
  std::vector<uint8_t> codes;            // T x n site-order Pauli codes
  std::vector<double> coeffs;            // T
  int nzwords = 0;                       // non-identity I/Z words (independent streams)
  // device copies
  DevGroup *d_groups = nullptr;
  DevNode *d_nodes = nullptr;
  double *d_leaf_coef = nullptr;
  int32_t *d_term_leaf = nullptr;
  uint64_t *d_zmask = nullptr;
  uint8_t *d_offdiag = nullptr;
  uint8_t *d_codes = nullptr;
  double *d_coeffs = nullptr;
  int32_t *d_sumidx_shared = nullptr;    // T: t for I/Z words, -1 for X/Y words
  int32_t *d_sumidx_word = nullptr;      // T: list position, -2 identity, -1 X/Y
  int32_t *d_wordlist = nullptr;         // nzwords word ids then nzwords last sites
  // Split evaluation at a cut site c (cut < 0: the prefix trie alone). Terms
  // ending before c close in the prefix trie's levels 0..c-1; the others pair a
  // prefix environment after site c-1 with a suffix environment of sites c..n-1
  // from a suffix trie (one 16 x 16 dot product per distinct pair).
  int cut = -1;
  std::vector<int32_t> term_slot;        // n x T: env slot of term t's prefix node at level s (-1 none);
                                         // released once the split plan is built
  std::vector<double> level_flops;       // prefix trie flops per level
  std::vector<DevGroup> sl_groups;       // prefix levels 0..cut-1 with split leaf ids
  std::vector<DevNode> sl_nodes;
  std::vector<int> sr_group_off, sr_node_off, sr_nslot;   // suffix levels, indexed by site (n + 1 / n)
  std::vector<DevGroup> sr_groups;
  std::vector<DevNode> sr_nodes;
  std::vector<int32_t> pairs;            // (prefix slot, suffix slot, leaf) per pair, by prefix slot
  std::vector<double> split_leaf_coef;
  std::vector<int32_t> split_term_leaf;
  int split_nleaf = 0, split_identity_leaf = -1, npairs = 0;
  int sl_max_slot = 1, sr_max_slot = 1;
  double split_flops = 0.0;
  long long split_node_sites = 0;
  DevGroup *d_sl_groups = nullptr, *d_sr_groups = nullptr;
  DevNode *d_sl_nodes = nullptr, *d_sr_nodes = nullptr;
  int32_t *d_pairs = nullptr, *d_split_term_leaf = nullptr;
  // Re(i^(prefix phase + suffix phase)) of every pair (pairs' order): the factor a
  // pair closure of two real-part environments takes (0 for an odd Y count)
  std::vector<double> pair_sign;
  double *d_pair_sign = nullptr;
  double *d_split_leaf_coef = nullptr;
  // Pair cotangents of the split gradient, summed in a fixed order: the pairs of
  // prefix slot j are pl_off[j] .. pl_off[j+1]-1 (pairs are sorted by prefix
  // slot); those of suffix slot r are pr_idx[pr_off[r] .. pr_off[r+1]-1].
  std::vector<int32_t> pl_off, pr_off, pr_idx;
  int32_t *d_pl_off = nullptr, *d_pr_off = nullptr, *d_pr_idx = nullptr;
  // Per-term cuts (energies; multicut_plan.inc): every word closes at its own
  // cut c_t, the prefix levels run 0..c_t-1 and the suffix levels c_t..l_t of it.
  // Levels keep their environments in per-level regions of one buffer per half
  // (region of level s: B x stride[s] slots from B x base[s]), since closures
  // read them at many levels. The gradient keeps the single-cut plan.
  bool mcut = false;                     // the current call uses the per-term-cut plan (select_plan)
  bool mc_pending = false, mc_built = false;
  // inputs kept for the deferred build: suffix-trie node of word t at site s
  // (n x T), suffix nodes per site, last sites, bond dims at load time
  std::vector<int32_t> mc_rslot, mc_sid_count;
  std::vector<int> mc_last, mc_bd;
  std::vector<int> mp_group_off, mp_node_off, mp_stride, mp_base;   // prefix levels 0 .. mp_levels - 1
  std::vector<DevGroup> mp_groups;
  std::vector<DevNode> mp_nodes;
  std::vector<int> ms_group_off, ms_node_off, ms_stride, ms_base;   // suffix levels, by site (n + 1 / n)
  std::vector<DevGroup> ms_groups;
  std::vector<DevNode> ms_nodes;
  std::vector<DevPair> mc_pairs;
  std::vector<double> mc_pair_sign, mc_leaf_coef;
  std::vector<int32_t> mc_term_leaf;
  int mp_levels = 0, ms_low = 0, mc_nleaf = 0, mc_identity_leaf = -1, mc_npairs = 0;
  long long mp_slots = 0, ms_slots = 0, mc_node_sites = 0, mc_groups_total = 0;
  int mc_max_slot = 1;
  double mc_flops = 0.0;
  DevGroup *d_mp_groups = nullptr, *d_ms_groups = nullptr;
  DevNode *d_mp_nodes = nullptr, *d_ms_nodes = nullptr;
  DevPair *d_mc_pairs = nullptr;
  double *d_mc_pair_sign = nullptr, *d_mc_leaf_coef = nullptr;
  int32_t *d_mc_term_leaf = nullptr;
  unsigned char *d_arena_mc = nullptr;   // the per-term-cut plan's device arrays
  // every d_ array above is a slice of this one device allocation
  unsigned char *d_arena = nullptr;
  ~Hamiltonian() { cudaFree(d_arena); cudaFree(d_arena_mc); }
  // leaves of the energy path (split plan when cut >= 0)
  int e_nleaf() const { return mcut ? mc_nleaf : cut >= 0 ? split_nleaf : nleaf; }
  int e_identity_leaf() const { return mcut ? mc_identity_leaf : cut >= 0 ? split_identity_leaf : identity_leaf; }
  const double *e_leaf_coef() const { return mcut ? d_mc_leaf_coef : cut >= 0 ? d_split_leaf_coef : d_leaf_coef; }
  const int32_t *e_term_leaf() const { return mcut ? d_mc_term_leaf : cut >= 0 ? d_split_term_leaf : d_term_leaf; }
};

// As-soon-as-possible schedule of a circuit's two-site gates for the K-CTA gate
// chains (evolve_pair_kernel: K = 2, evolve_quad_real_kernel: K = 4), at most K
// gates per step on disjoint site pairs (step t: sched[K t .. K t + K - 1]), and
// the one-site gates each two-site gate folds in (see EvolveParams); the folding
// does not depend on K.
struct PairSched {
  std::vector<int32_t> sched, gate_q, qlist, tail_off;
  int nsteps = 0;
};

// Which factor of each two-site gate carries the singular values (a gauge choice,
// see evolve.cuh): the left one when the next two-site gate that touches either
// of its sites touches only its right site, else the right one (the reference's
// packing). Leaves every one-site gate's flags at 0.
void mark_sigma_side(std::vector<DevGate> &gates) {
  for (size_t i = 0; i < gates.size(); ++i) {
    if (gates[i].kind != GATE_TWO) continue;
    const int s = gates[i].site;
    int flags = 0;
    for (size_t j = i + 1; j < gates.size(); ++j) {
      if (gates[j].kind != GATE_TWO) continue;
      const int t = gates[j].site;                  // touches t and t + 1
      const bool left = (t == s || t + 1 == s), right = (t == s + 1 || t + 1 == s + 1);
      if (!left && !right) continue;
      flags = (right && !left) ? GATE_SIGMA_LEFT : 0;
      break;
    }
    gates[i].flags = flags;
  }
}

PairSched build_pair_schedule(const std::vector<DevGate> &gates, int n, int K = 2) {
  PairSched ps;
  ps.gate_q.assign(4 * std::max<size_t>(gates.size(), 1), 0);
  std::vector<std::vector<int32_t>> pend(n);
  std::vector<int> last_step(n, -1), count;
  for (int gi = 0; gi < (int)gates.size(); ++gi) {
    const DevGate &g = gates[gi];
    if (g.kind == GATE_ONE) {
      pend[g.site].push_back(gi);
      continue;
    }
    const int s = g.site;
    for (int side = 0; side < 2; ++side) {
      ps.gate_q[4 * gi + 2 * side] = (int32_t)ps.qlist.size();
      ps.qlist.insert(ps.qlist.end(), pend[s + side].begin(), pend[s + side].end());
      ps.gate_q[4 * gi + 2 * side + 1] = (int32_t)ps.qlist.size();
      pend[s + side].clear();
    }
    int t = std::max(last_step[s], last_step[s + 1]) + 1;
    while (t < (int)count.size() && count[t] >= K) ++t;
    if (t == (int)count.size()) {
      count.push_back(0);
      ps.sched.insert(ps.sched.end(), K, -1);
    }
    ps.sched[K * t + count[t]] = gi;
    ++count[t];
    last_step[s] = last_step[s + 1] = t;
  }
  ps.tail_off.resize(n + 1);
  for (int x = 0; x < n; ++x) {
    ps.tail_off[x] = (int32_t)ps.qlist.size();
    ps.qlist.insert(ps.qlist.end(), pend[x].begin(), pend[x].end());
  }
  ps.tail_off[n] = (int32_t)ps.qlist.size();
  ps.nsteps = (int)count.size();
  return ps;
}

// A partition set: K independent circuits with their own widths, parameters
// and Hamiltonians, evaluated together in one batch. Per-partition tables sit
// at fixed strides (widest partition, most terms, most leaves); the trie
// levels of all partitions are merged level by level, so one launch per level
// runs every partition's own plan through a work list.
struct PartSet {
  int K = 0, n_max = 0, P_max = 0, T_max = 1, leaf_stride = 1, W = 1;
  int site_order = 0;
  bool all_diagonal = true;
  bool real = true;                     // every partition's circuit of real gates
  bool mixed = false;                   // some real, some complex: the per-partition chain kernels
  int32_t *d_part_real = nullptr;       // K flags (mixed sets)
  cplx init0, init1;
  std::vector<int32_t> part_n, part_P, part_T, part_nleaf, part_idleaf, part_gate_off;
  std::vector<int> lvl_group_off, lvl_node_off, lvl_nslot;   // merged levels (n_max + 1 / n_max)
  std::vector<int32_t> lvl_pg_begin, lvl_pg_count;           // [s * K + k]: partition k's groups in level s
  int nlevels = 0;
  double flops = 0.0;                                        // one evaluation of every partition
  std::vector<int> bonds;                                    // K x (n_max + 1) allocation bounds
  DevGate *d_gates = nullptr;
  cplx *d_mats = nullptr;
  DevGroup *d_groups = nullptr;
  DevNode *d_nodes = nullptr;
  PairSched psched;                 // merged two-CTA schedules
  std::vector<int32_t> step_off, part_tail_off;
  int32_t *d_sched = nullptr, *d_step_off = nullptr, *d_gate_q = nullptr, *d_qlist = nullptr;
  int32_t *d_tail_off = nullptr, *d_part_tail_off = nullptr;
  int32_t *d_part = nullptr;        // part_n | part_T | part_nleaf | part_idleaf | part_gate_off (K+1)
  double *d_leaf_coef = nullptr;    // K x leaf_stride
  int32_t *d_term_leaf = nullptr;   // K x T_max
  uint64_t *d_zmask = nullptr;      // K x T_max x W
  double *d_coeffs = nullptr;       // K x T_max
  int32_t *d_sumidx = nullptr;      // K x T_max: t for I/Z words, -1 for X/Y words
  // per-copies cache: state -> partition map and the level work lists
  int cached_copies = 0;
  std::vector<int> work_off;        // nlevels + 1 (items)
  int32_t *d_st_part = nullptr;
  int32_t *d_work = nullptr;
  ~PartSet() {
    cudaFree(d_gates); cudaFree(d_mats); cudaFree(d_groups); cudaFree(d_nodes); cudaFree(d_part);
    cudaFree(d_leaf_coef); cudaFree(d_term_leaf); cudaFree(d_zmask); cudaFree(d_coeffs);
    cudaFree(d_sumidx); cudaFree(d_st_part); cudaFree(d_work);
    cudaFree(d_sched); cudaFree(d_step_off); cudaFree(d_gate_q); cudaFree(d_qlist); cudaFree(d_tail_off);
    cudaFree(d_part_tail_off); cudaFree(d_part_real);
  }
};

template <typename T>
struct DevBuf {
  T *ptr = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t count) {
    if (count <= cap) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr; cap = 0;
    cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) cap = count;
    return e;
  }
  void release() { if (ptr) cudaFree(ptr); ptr = nullptr; cap = 0; }
};

}  // namespace

// Trie-level kernel variants (the autotuner's candidates).
enum : int {
  LV_SIMT4 = 0, LV_MMA4 = 1, LV_MMA8 = 2, LV_PF4 = 3, LV_MMAPF4 = 4, LV_MMA3PF4 = 5,
  LV_REALPF4 = 6,   // real arithmetic: circuits of real gates only
  LV_COUNT = 7
};

struct vqemps_ctx {
  int device = 0;
  int max_bond = 16;
  double abs_cut = 0.0, rel_cut = 0.0;
  std::string err;
  // circuit
  int n = 0, P = 0, site_order = 0;
  bool have_circuit = false;
  // every gate real (and the initial state real): the states have real
  // amplitudes and the real-arithmetic level kernels may run
  bool real_circuit = false;
  bool doubling_ok = false;             // only adjacent CX two-qubit gates (gradient path)
  std::vector<DevGate> gates;
  std::vector<cplx> mats;
  std::vector<int> bonds;               // zero-cutoff allocation bound, n + 1
  std::vector<int> site_of_qubit;
  cplx init0, init1;
  std::vector<GradOp> grad_ops;         // op list of the bond-doubling (gradient) path
  std::vector<SiteEvent> site_events;   // per-site event lists (gradient path)
  std::vector<int32_t> ev_off, ev_dims, slot_off, slot_list;
  int nslots = 0;
  DevGate *d_gates = nullptr;
  cplx *d_mats = nullptr;
  SiteEvent *d_events = nullptr;
  int32_t *d_ev_off = nullptr, *d_ev_dims = nullptr, *d_slot_off = nullptr, *d_slot_list = nullptr;
  // hamiltonians
  std::map<int, std::unique_ptr<Hamiltonian>> hams;
  std::map<int, std::unique_ptr<PartSet>> parts;
  int next_handle = 1;
  // workspaces
  DevBuf<cplx> sites, right, env0, env1, env2, env3, sites_t;
  DevBuf<int32_t> bonds_ws, status;
  DevBuf<double> leafval, theta_stage, energy_stage, per_term_stage;
  DevBuf<double> panels, panels_t, right_real;   // real-arithmetic levels: real site panels, real R
  bool right_real_fresh = false;        // right_real holds the last launch_right's environments
  bool panels_fresh = false;            // ... and panels (panels_t too when panels_t_fresh) its site panels
  bool panels_t_fresh = false;
  DevBuf<cplx> mflat_p, mflat_s;        // per-term-cut plan: level regions of the prefix / suffix half
  int level_launches = 0;               // kernels the last run_levels launched
  int evolve_launches = 0;              // kernels the last launch_evolve launched
  DevBuf<cplx> upend;                   // pending one-site products of the multi-CTA chains
  // The split evaluation's suffix half runs on a second stream, forked from and
  // joined back into the caller's stream (so graph capture sees both).
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  DevBuf<uint64_t> bits, seeds;
  DevBuf<int32_t> zsum;
  DevBuf<cplx> branch;
  DevBuf<double> analytic_stage;
  DevBuf<cplx> grad_sites, grad_envs, grad_seg, grad_bar0, grad_bar1, grad_sitebar, grad_partial, grad_leafsum;
  // split gradient: transposed sites, suffix environments (all levels), suffix
  // cotangents (ping-pong), cotangents of R_{s+1} from the suffix roots, the
  // suffix backward's site partials (it runs beside the prefix half on the
  // second stream) and the left sweep's F at the cut
  DevBuf<cplx> grad_sites_t, grad_senv, grad_sbar0, grad_sbar1, grad_rootbar, grad_partial_s, grad_fstate;
  DevBuf<double> grad_stage;
  int last_B = 0;
  int forced_variant = -1;              // level kernel variant, -1: autotune
  // Autotuner decisions shared by plans of one size class: (batch-size bucket,
  // split or prefix plan, power-of-two bucket of node-sites) -> variant.
  std::map<int, int> tuned_by_shape;
  int grad_checkpoint = 8;              // gradient: keep every 8th level's environments
  int grad_mma = 2;                     // gradient levels: 0 SIMT, 1 FP64 DMMA, 2 DMMA with Gauss forward
  int split_mode = -1;                  // split evaluation: -1 when it saves work, 0 never, 1 always
  int evolve_pair = -1;                 // gate chain: 2 four-CTA clusters (real circuits), 1 two-CTA
                                        // clusters, 0 one CTA, -1 by batch size
  int sm_count = 148;
  PairSched psched;
  int32_t *d_sched = nullptr, *d_gate_q = nullptr, *d_qlist = nullptr, *d_tail_off = nullptr;
  int32_t *d_qsched = nullptr;          // four gates per step (evolve_quad_real_kernel)
  int qsteps = 0;
  int quad_clusters = -1;               // clusters of evolve_quad_real_kernel the GPU holds at once (-1: not queried)
  ~vqemps_ctx() {
    cudaFree(d_gates); cudaFree(d_mats); cudaFree(d_events); cudaFree(d_ev_off);
    cudaFree(d_ev_dims); cudaFree(d_slot_off); cudaFree(d_slot_list);
    cudaFree(d_sched); cudaFree(d_gate_q); cudaFree(d_qlist); cudaFree(d_tail_off); cudaFree(d_qsched);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (aux) cudaStreamDestroy(aux);
  }
};

static int fail(vqemps_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return code;
}

#define CUDA_TRY(ctx, expr)                                                          \
  do {                                                                               \
    cudaError_t _e = (expr);                                                         \
    if (_e != cudaSuccess)                                                           \
      return fail(ctx, VQEMPS_CUDA_ERROR, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

static cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }
static bool build_site_events(vqemps_ctx *ctx);
static int upload_site_events(vqemps_ctx *ctx);

// ---------------------------------------------------------------------------
// creation
// ---------------------------------------------------------------------------
extern "C" int vqemps_create(int device, int max_bond, double abs_cut, double rel_cut,
                             vqemps_ctx **out) {
  if (!out) return VQEMPS_INVALID;
  *out = nullptr;
  if (max_bond < 1 || max_bond > CHI) return VQEMPS_INVALID;
  if (!(abs_cut >= 0.0) || !(rel_cut >= 0.0)) return VQEMPS_INVALID;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
    return VQEMPS_CUDA_ERROR;
  if (cudaSetDevice(device) != cudaSuccess) return VQEMPS_CUDA_ERROR;
  auto *ctx = new vqemps_ctx();
  ctx->device = device;
  ctx->max_bond = max_bond;
  ctx->abs_cut = abs_cut;
  ctx->rel_cut = rel_cut;
  cudaFuncSetAttribute(evolve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(evolve_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(evolve_real_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(evolve_pair_real_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(evolve_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(evolve_pair_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (const char *v = std::getenv("VQEMPS_EVOLVE"))
    ctx->evolve_pair = std::strcmp(v, "chain") == 0 ? 0 : std::strcmp(v, "pair") == 0 ? 1
                       : std::strcmp(v, "quad") == 0 ? 2 : -1;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  cudaFuncSetAttribute(level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(LevelSmem));
  cudaFuncSetAttribute(level_mma_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(LevelMmaSmem<4>));
  cudaFuncSetAttribute(level_mma_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(LevelMmaSmem<8>));
  cudaFuncSetAttribute(level_pf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(LevelPfSmem));
  cudaFuncSetAttribute(level_mma_pf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(LevelMmaPfSmem));
  cudaFuncSetAttribute(level_mma3_pf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(LevelMmaPfSmem));
  grad_set_attributes();
  cudaFuncSetAttribute(grad_fwd_level_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(GradFwdMmaSmem));
  cudaFuncSetAttribute(grad_bwd_level_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(GradBwdMmaSmem));
  cudaFuncSetAttribute(grad_fwd_level_mma3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(GradFwdMmaSmem));
  cudaFuncSetAttribute(grad_fwd_level_real_a_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(GradFwdRealSmem));
  cudaFuncSetAttribute(grad_bwd_level_real_a_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(GradBwdRealSmem));
  if (const char *v = std::getenv("VQEMPS_GRAD_VARIANT"))
    ctx->grad_mma = std::strcmp(v, "simt") == 0 ? 0 : std::strcmp(v, "dmma") == 0 ? 1 : 2;
  // VQEMPS_LEVEL_VARIANT pins the trie-level kernel (a name or an index); the
  // autotuner's timings are meaningless under a serialising profiler.
  if (const char *v = std::getenv("VQEMPS_LEVEL_VARIANT")) {
    static const char *names[LV_COUNT] = {"simt", "dmma4", "dmma8", "simt_pf", "dmma_pf", "dmma3_pf", "real_pf"};
    for (int i = 0; i < LV_COUNT; ++i)
      if (std::strcmp(v, names[i]) == 0 || (v[0] == '0' + i && v[1] == 0)) ctx->forced_variant = i;
  }
  *out = ctx;
  return VQEMPS_OK;
}

extern "C" int vqemps_destroy(vqemps_ctx *ctx) {
  if (!ctx) return VQEMPS_OK;
  cudaSetDevice(ctx->device);
  ctx->hams.clear();
  ctx->parts.clear();
  ctx->sites.release(); ctx->right.release(); ctx->env0.release(); ctx->env1.release();
  ctx->env2.release(); ctx->env3.release(); ctx->sites_t.release();
  ctx->bonds_ws.release(); ctx->status.release(); ctx->leafval.release();
  ctx->theta_stage.release(); ctx->energy_stage.release(); ctx->per_term_stage.release();
  ctx->bits.release(); ctx->zsum.release(); ctx->seeds.release(); ctx->branch.release();
  ctx->analytic_stage.release();
  ctx->grad_sites.release(); ctx->grad_envs.release(); ctx->grad_bar0.release();
  ctx->grad_bar1.release(); ctx->grad_sitebar.release(); ctx->grad_stage.release();
  ctx->grad_partial.release(); ctx->grad_leafsum.release(); ctx->grad_seg.release();
  ctx->grad_sites_t.release(); ctx->grad_senv.release(); ctx->grad_sbar0.release();
  ctx->grad_sbar1.release(); ctx->grad_rootbar.release(); ctx->grad_partial_s.release();
  ctx->grad_fstate.release();
  delete ctx;
  return VQEMPS_OK;
}

extern "C" const char *vqemps_last_error(const vqemps_ctx *ctx) {
  if (!ctx) return "null context";
  return ctx->err.c_str();
}

// ---------------------------------------------------------------------------
// circuit compilation
// ---------------------------------------------------------------------------
static void push_matrix(std::vector<cplx> &mats, const cplx *m, int count, int *offset) {
  *offset = (int)mats.size();
  for (int i = 0; i < count; ++i) mats.push_back(m[i]);
}

extern "C" int vqemps_set_circuit(vqemps_ctx *ctx, int n, const vqemps_op *ops, int nops,
                                  const double *matrices, int nmatrices, int initial,
                                  int site_order) {
  if (!ctx) return VQEMPS_INVALID;
  if (n < 2) return fail(ctx, VQEMPS_INVALID, "the MPS engine needs >= 2 qubits");
  if (nops < 0 || (nops > 0 && !ops)) return fail(ctx, VQEMPS_INVALID, "bad op list");
  if (nmatrices < 0 || (nmatrices > 0 && !matrices)) return fail(ctx, VQEMPS_INVALID, "bad matrix table");
  if (site_order != 0 && site_order != 1) return fail(ctx, VQEMPS_INVALID, "site_order must be 0 or 1");
  if (EvolveSmem::bytes(n) > 200 * 1024) return fail(ctx, VQEMPS_INVALID, "too many qubits for one CTA");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const double r2 = 1.0 / std::sqrt(2.0);
  cplx init0, init1;
  switch (initial) {
    case VQEMPS_INIT_ZERO: init0 = cmake(1, 0); init1 = cmake(0, 0); break;
    case VQEMPS_INIT_ONE: init0 = cmake(0, 0); init1 = cmake(1, 0); break;
    case VQEMPS_INIT_PLUS: init0 = cmake(r2, 0); init1 = cmake(r2, 0); break;
    case VQEMPS_INIT_MINUS: init0 = cmake(r2, 0); init1 = cmake(-r2, 0); break;
    default: return fail(ctx, VQEMPS_INVALID, "unknown initial state");
  }
  std::vector<int> site_of(n);
  for (int q = 0; q < n; ++q) site_of[q] = site_order == 1 ? n - 1 - q : q;

  std::vector<cplx> mats;
  // fixed one-site matrices: H X Y Z S SDG
  int fixed_off[6];
  {
    const cplx h[4] = {cmake(r2, 0), cmake(r2, 0), cmake(r2, 0), cmake(-r2, 0)};
    const cplx x[4] = {cmake(0, 0), cmake(1, 0), cmake(1, 0), cmake(0, 0)};
    const cplx y[4] = {cmake(0, 0), cmake(0, -1), cmake(0, 1), cmake(0, 0)};
    const cplx z[4] = {cmake(1, 0), cmake(0, 0), cmake(0, 0), cmake(-1, 0)};
    const cplx sg[4] = {cmake(1, 0), cmake(0, 0), cmake(0, 0), cmake(0, 1)};
    const cplx sd[4] = {cmake(1, 0), cmake(0, 0), cmake(0, 0), cmake(0, -1)};
    push_matrix(mats, h, 4, &fixed_off[0]);
    push_matrix(mats, x, 4, &fixed_off[1]);
    push_matrix(mats, y, 4, &fixed_off[2]);
    push_matrix(mats, z, 4, &fixed_off[3]);
    push_matrix(mats, sg, 4, &fixed_off[4]);
    push_matrix(mats, sd, 4, &fixed_off[5]);
  }
  int swap_off;
  {
    cplx sw[16];
    for (int I = 0; I < 2; ++I)
      for (int J = 0; J < 2; ++J)
        for (int i = 0; i < 2; ++i)
          for (int j = 0; j < 2; ++j)
            sw[(I * 2 + J) * 4 + (i * 2 + j)] = cmake((I == j && J == i) ? 1 : 0, 0);
    push_matrix(mats, sw, 16, &swap_off);
  }
  std::vector<DevGate> gates;
  std::vector<GradOp> gops;
  std::vector<int> bonds(n + 1, 1);
  int P = 0;
  bool doubling_ok = true;
  bool real = true;        // RY, H, X, Z, CX, SWAP and real U1 / U2 matrices keep amplitudes real
  const int maxb = ctx->max_bond;
  auto add_two = [&](int s, int mat) {
    DevGate g{};
    g.kind = GATE_TWO; g.site = s; g.mat = mat; g.rot = ROT_NONE; g.param = -1; g.angle = 0;
    gates.push_back(g);
    bonds[s + 1] = std::min(std::min(2 * bonds[s], 2 * bonds[s + 2]), maxb);
  };
  for (int k = 0; k < nops; ++k) {
    const vqemps_op &op = ops[k];
    auto bad_q = [&](int q) { return q < 0 || q >= n; };
    if (op.kind <= VQEMPS_SDG || op.kind == VQEMPS_U1) {
      if (bad_q(op.q0)) return fail(ctx, VQEMPS_INVALID, "qubit index out of range");
      DevGate g{};
      g.kind = GATE_ONE; g.site = site_of[op.q0]; g.param = -1; g.angle = op.angle;
      g.mat = -1; g.rot = ROT_NONE;
      GradOp go{};
      go.kind = GOP_ONE; go.site = g.site; go.param = -1; go.angle = op.angle; go.mat = -1;
      go.rot = ROT_NONE;
      if (op.kind == VQEMPS_RX || op.kind == VQEMPS_RZ || op.kind == VQEMPS_Y || op.kind == VQEMPS_S ||
          op.kind == VQEMPS_SDG)
        real = false;
      if (op.kind <= VQEMPS_RZ) {
        g.rot = op.kind == VQEMPS_RX ? ROT_X : op.kind == VQEMPS_RY ? ROT_Y : ROT_Z;
        g.param = op.param;
        if (op.param >= 0) P = std::max(P, op.param + 1);
        go.rot = g.rot; go.param = g.param;
      } else if (op.kind == VQEMPS_U1) {
        if (op.matrix < 0 || op.matrix + 4 > nmatrices)
          return fail(ctx, VQEMPS_INVALID, "U1 matrix index out of range");
        cplx m[4];
        for (int i = 0; i < 4; ++i) m[i] = cmake(matrices[2 * (op.matrix + i)], matrices[2 * (op.matrix + i) + 1]);
        for (int i = 0; i < 4; ++i)
          if (m[i].y != 0.0) real = false;
        push_matrix(mats, m, 4, &g.mat);
        go.mat = g.mat;
      } else {
        g.mat = fixed_off[op.kind - VQEMPS_H];
        go.mat = g.mat;
      }
      gates.push_back(g);
      gops.push_back(go);
      continue;
    }
    if (op.kind != VQEMPS_CX && op.kind != VQEMPS_U2 && op.kind != VQEMPS_SWAP)
      return fail(ctx, VQEMPS_INVALID, "unsupported gate kind (>2-qubit or multi-control gates are not supported)");
    if (bad_q(op.q0) || bad_q(op.q1) || op.q0 == op.q1)
      return fail(ctx, VQEMPS_INVALID, "bad two-qubit gate operands");
    cplx g4[16];
    if (op.kind == VQEMPS_CX) {
      // controlledGate (simulator_mps_dist.cu:376-384): [(C*2+T)*4 + (c*2+t)]
      for (int C = 0; C < 2; ++C)
        for (int T = 0; T < 2; ++T)
          for (int c = 0; c < 2; ++c)
            for (int t = 0; t < 2; ++t) {
              double v = 0;
              if (C == c) v = (c == 0) ? (T == t ? 1 : 0) : (T != t ? 1 : 0);
              g4[(C * 2 + T) * 4 + (c * 2 + t)] = cmake(v, 0);
            }
    } else if (op.kind == VQEMPS_SWAP) {
      for (int i = 0; i < 16; ++i) g4[i] = mats[swap_off + i];
    } else {
      if (op.matrix < 0 || op.matrix + 16 > nmatrices)
        return fail(ctx, VQEMPS_INVALID, "U2 matrix index out of range");
      for (int i = 0; i < 16; ++i) {
        g4[i] = cmake(matrices[2 * (op.matrix + i)], matrices[2 * (op.matrix + i) + 1]);
        if (g4[i].y != 0.0) real = false;
      }
    }
    int a = site_of[op.q0], bsite = site_of[op.q1];
    if (a > bsite) {  // swapOperands (sharded_mps.cuh:555-562)
      cplx h4[16];
      for (int I = 0; I < 2; ++I)
        for (int J = 0; J < 2; ++J)
          for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j)
              h4[(I * 2 + J) * 4 + (i * 2 + j)] = g4[(J * 2 + I) * 4 + (j * 2 + i)];
      std::memcpy(g4, h4, sizeof(g4));
      std::swap(a, bsite);
    }
    int off;
    push_matrix(mats, g4, 16, &off);
    // SWAP routing (sharded_mps.cuh:565-572)
    for (int x = bsite; x > a + 1; --x) add_two(x - 1, swap_off);
    add_two(a, off);
    for (int x = a + 1; x < bsite; ++x) add_two(x, swap_off);
    if (op.kind == VQEMPS_CX && bsite == a + 1) {
      GradOp go{};
      go.kind = GOP_CX; go.site = a;
      go.param = (site_of[op.q0] == a) ? 0 : 1;   // 0: control on the left site
      go.mat = -1; go.rot = ROT_NONE; go.angle = 0;
      gops.push_back(go);
    } else {
      doubling_ok = false;
    }
  }
  mark_sigma_side(gates);
  // upload
  cudaFree(ctx->d_gates); ctx->d_gates = nullptr;
  cudaFree(ctx->d_mats); ctx->d_mats = nullptr;
  CUDA_TRY(ctx, cudaMalloc(&ctx->d_gates, std::max<size_t>(gates.size(), 1) * sizeof(DevGate)));
  CUDA_TRY(ctx, cudaMalloc(&ctx->d_mats, std::max<size_t>(mats.size(), 1) * sizeof(cplx)));
  if (!gates.empty())
    CUDA_TRY(ctx, cudaMemcpy(ctx->d_gates, gates.data(), gates.size() * sizeof(DevGate), cudaMemcpyHostToDevice));
  CUDA_TRY(ctx, cudaMemcpy(ctx->d_mats, mats.data(), mats.size() * sizeof(cplx), cudaMemcpyHostToDevice));
  {
    PairSched ps = build_pair_schedule(gates, n);
    auto upi = [&](int32_t *&dst, const std::vector<int32_t> &v) -> cudaError_t {
      cudaFree(dst);
      dst = nullptr;
      cudaError_t e = cudaMalloc(&dst, std::max<size_t>(v.size(), 1) * sizeof(int32_t));
      if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(dst, v.data(), v.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
      return e;
    };
    CUDA_TRY(ctx, upi(ctx->d_sched, ps.sched));
    CUDA_TRY(ctx, upi(ctx->d_gate_q, ps.gate_q));
    CUDA_TRY(ctx, upi(ctx->d_qlist, ps.qlist));
    CUDA_TRY(ctx, upi(ctx->d_tail_off, ps.tail_off));
    ctx->psched = std::move(ps);
    const PairSched qs = build_pair_schedule(gates, n, 4);
    CUDA_TRY(ctx, upi(ctx->d_qsched, qs.sched));
    ctx->qsteps = qs.nsteps;
  }
  ctx->gates = std::move(gates);
  ctx->mats = std::move(mats);
  ctx->grad_ops = std::move(gops);
  ctx->bonds = bonds;
  ctx->n = n;
  ctx->quad_clusters = -1;
  ctx->P = P;
  ctx->site_order = site_order;
  ctx->site_of_qubit = site_of;
  ctx->init0 = init0;
  ctx->init1 = init1;
  ctx->doubling_ok = doubling_ok;
  ctx->have_circuit = true;
  ctx->real_circuit = real;
  if (ctx->doubling_ok) ctx->doubling_ok = build_site_events(ctx);
  if (ctx->doubling_ok) {
    const int rc = upload_site_events(ctx);
    if (rc) return rc;
  }
  // Hamiltonians are bound to a width and site order: drop stale ones.
  for (auto it = ctx->hams.begin(); it != ctx->hams.end();) {
    if (it->second->n != n) it = ctx->hams.erase(it);
    else ++it;
  }
  return VQEMPS_OK;
}

extern "C" int vqemps_num_params(const vqemps_ctx *ctx, int *params) {
  if (!ctx || !params || !ctx->have_circuit) return VQEMPS_INVALID;
  *params = ctx->P;
  return VQEMPS_OK;
}

extern "C" int vqemps_bond_dims(const vqemps_ctx *ctx, int *dims) {
  if (!ctx || !dims || !ctx->have_circuit) return VQEMPS_INVALID;
  for (int i = 0; i <= ctx->n; ++i) dims[i] = ctx->bonds[i];
  return VQEMPS_OK;
}

#include "multicut_plan.inc"
#include "split_plan.inc"

// ---------------------------------------------------------------------------
// Hamiltonian plan: one prefix trie over the sorted site-order words, each path
// cut after its term's last non-identity site.
// ---------------------------------------------------------------------------
extern "C" int vqemps_set_hamiltonian(vqemps_ctx *ctx, const char *words, const double *coeffs,
                                      int T, int *handle) {
  if (!ctx || !handle) return VQEMPS_INVALID;
  if (!ctx->have_circuit) return fail(ctx, VQEMPS_INVALID, "set a circuit before a Hamiltonian");
  if (T < 0 || (T > 0 && (!words || !coeffs))) return fail(ctx, VQEMPS_INVALID, "bad word list");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int n = ctx->n;
  auto h = std::make_unique<Hamiltonian>();
  h->n = n;
  h->T = T;
  // site-order codes (buildPauliTermData reverses words for the msb map)
  std::vector<uint8_t> code((size_t)T * n);
  std::vector<int> last(T, -1);
  const int W = (n + 63) / 64;
  h->zmask.assign((size_t)T * W, 0);
  h->offdiag.assign(T, 0);
  for (int t = 0; t < T; ++t) {
    for (int q = 0; q < n; ++q) {
      const char c = words[(size_t)t * n + q];
      uint8_t v;
      switch (c) {
        case 'I': v = 0; break;
        case 'X': v = 1; break;
        case 'Y': v = 2; break;
        case 'Z': v = 3; break;
        default: return fail(ctx, VQEMPS_INVALID, "Invalid analytic Pauli");
      }
      const int s = ctx->site_of_qubit[q];
      code[(size_t)t * n + s] = v;
      if (v == 3) h->zmask[(size_t)t * W + q / 64] |= (1ULL << (q % 64));
      if (v == 1 || v == 2) h->offdiag[t] = 1;
    }
    for (int s = n - 1; s >= 0; --s)
      if (code[(size_t)t * n + s] != 0) { last[t] = s; break; }
    if (!std::isfinite(coeffs[t])) return fail(ctx, VQEMPS_INVALID, "nonfinite coefficient");
    if (h->offdiag[t]) h->all_diagonal = false;
  }
  h->coeffs.assign(coeffs, coeffs + T);
  std::vector<int32_t> sumidx_shared(T), sumidx_word(T), wl, wlast;
  for (int t = 0; t < T; ++t) {
    sumidx_shared[t] = h->offdiag[t] ? -1 : t;
    if (h->offdiag[t]) { sumidx_word[t] = -1; continue; }
    if (last[t] < 0) { sumidx_word[t] = -2; continue; }
    sumidx_word[t] = (int32_t)wl.size();
    wl.push_back(t);
    wlast.push_back(last[t]);
  }
  h->nzwords = (int)wl.size();
  wl.insert(wl.end(), wlast.begin(), wlast.end());
  std::vector<int> order(T);
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    const int c = std::memcmp(&code[(size_t)a * n], &code[(size_t)b * n], n);
    return c != 0 ? c < 0 : a < b;
  });
  h->term_leaf.assign(T, -1);
  // identity words close against the norm
  for (int t = 0; t < T; ++t)
    if (last[t] < 0) {
      if (h->identity_leaf < 0) {
        h->identity_leaf = h->nleaf++;
        h->leaf_coef.push_back(0.0);
        h->leaf_level.push_back(-1);
      }
      h->term_leaf[t] = h->identity_leaf;
      h->leaf_coef[h->identity_leaf] += coeffs[t];
    }
  // the split plan's suffix trie needs only the words: build it on a second host
  // thread while this one builds the prefix trie
  const bool want_split = ctx->split_mode != 0 && n >= 3 && T > 0;
  std::future<SuffixTrie> suffix;
  if (want_split)
    suffix = std::async(std::launch::async, build_suffix_trie, n, T, std::cref(code), std::cref(last),
                        std::cref(ctx->bonds));
  // level-by-level construction over the sorted order
  std::vector<int> active;  // words (sorted order) still on a path at this level
  for (int t : order)
    if (last[t] >= 0) active.push_back(t);
  std::vector<int> parent_node(active.size(), -1);   // node id at the previous level
  std::vector<int> prev_slot;                        // env slot of each node of the previous level
  std::vector<int> prev_phase;                       // Y-count phase of each node of the previous level
  h->group_off.assign(n + 1, 0);
  h->node_off.assign(n + 1, 0);
  h->nslot.assign(n, 0);
  h->term_slot.assign((size_t)n * T, -1);   // level-major: one level's writes stay in one row
  h->level_flops.assign(n, 0.0);
  const std::vector<int> &bd = ctx->bonds;
  for (int s = 0; s < n; ++s) {
    h->group_off[s] = (int)h->groups.size();
    h->node_off[s] = (int)h->nodes.size();
    std::vector<int> next_active, next_parent;
    std::vector<int> node_has_child;
    int level_nodes = 0;
    int prev_parent = -2, prev_code = -1, cur_node = -1;
    // pass 1: node assignment (consecutive words with equal (parent, code) share a node)
    std::vector<int> node_of(active.size());
    for (size_t j = 0; j < active.size(); ++j) {
      const int t = active[j];
      const int c = code[(size_t)t * n + s];
      if (parent_node[j] != prev_parent || c != prev_code) {
        cur_node = level_nodes++;
        DevNode nd{};
        nd.code = c; nd.env_slot = -1; nd.leaf = -1;
        nd.phase = ((s == 0 ? 0 : prev_phase[parent_node[j]]) + (c == 2 ? 1 : 0)) & 3;
        h->nodes.push_back(nd);
        node_has_child.push_back(0);
        prev_parent = parent_node[j];
        prev_code = c;
      }
      node_of[j] = cur_node;
      DevNode &nd = h->nodes[h->node_off[s] + cur_node];
      if (last[t] == s) {
        if (nd.leaf < 0) {
          nd.leaf = h->nleaf++;
          h->leaf_coef.push_back(0.0);
          h->leaf_level.push_back(s);
        }
        h->term_leaf[t] = nd.leaf;
        h->leaf_coef[nd.leaf] += coeffs[t];
      } else {
        node_has_child[cur_node] = 1;
        next_active.push_back(t);
        next_parent.push_back(cur_node);
      }
    }
    // env slots for nodes with descendants
    int slots = 0;
    std::vector<int> slot_of(level_nodes, -1);
    for (int k = 0; k < level_nodes; ++k)
      if (node_has_child[k]) {
        slot_of[k] = slots++;
        h->nodes[h->node_off[s] + k].env_slot = slot_of[k];
      }
    h->nslot[s] = slots;
    for (size_t j = 0; j < active.size(); ++j) h->term_slot[(size_t)s * T + active[j]] = slot_of[node_of[j]];
    h->max_slot = std::max(h->max_slot, slots);
    // groups: consecutive nodes with the same parent
    {
      size_t j = 0;
      while (j < active.size()) {
        const int par = parent_node[j];
        const int first = node_of[j];
        int lastn = first;
        while (j < active.size() && parent_node[j] == par) { lastn = node_of[j]; ++j; }
        DevGroup g{};
        g.parent_slot = (s == 0) ? -1 : prev_slot[par];
        g.child_begin = first;
        g.nchild = lastn - first + 1;
        g.classes = 0;
        for (int k = first; k <= lastn; ++k) {
          const int c = h->nodes[h->node_off[s] + k].code;
          g.classes |= (c == 0 || c == 3) ? 1 : 2;
        }
        {
          const DevNode &c0 = h->nodes[h->node_off[s] + first];
          if ((c0.phase - (c0.code == 2 ? 1 : 0)) & 1) g.classes |= 4;   // odd parent phase
        }
        h->groups.push_back(g);
        // flop accounting with the actual bond dims (dl x dr site), as the
        // prefetch DMMA level kernels execute it: the children are Hermitian, so
        // the I/Z products form three of four output tiles and the X/Y pair one
        // product (t1 = t0^H)
        const double dl = bd[s], dr = bd[s + 1];
        const double gf = 8.0 * 2.0 * dl * dl * dr                                 // S_i = E A_i
                          + ((g.classes & 1) ? 0.75 : 0.0) * 8.0 * 2.0 * dl * dr * dr  // I/Z products
                          + ((g.classes & 2) ? 0.5 : 0.0) * 8.0 * 2.0 * dl * dr * dr;  // X/Y product
        h->flops += gf;
        h->level_flops[s] += gf;
        h->flops_survey += (lastn - first + 1) * 16.0 * dl * dr * (dl + dr);
        h->node_sites += lastn - first + 1;
      }
    }
    prev_slot = slot_of;
    prev_phase.resize(level_nodes);
    for (int k = 0; k < level_nodes; ++k) prev_phase[k] = h->nodes[h->node_off[s] + k].phase;
    active.swap(next_active);
    parent_node.swap(next_parent);
  }
  h->group_off[n] = (int)h->groups.size();
  h->node_off[n] = (int)h->nodes.size();
  build_split_plan(*h, want_split ? suffix.get() : SuffixTrie{}, code, last, ctx->bonds, ctx->split_mode);
  std::vector<int32_t>().swap(h->term_slot);
  // upload: every plan array is a 256-byte aligned slice of ONE device
  // allocation, filled by one copy of a packed host image (tens of separate
  // allocations and copies cost more than the plan build itself at 40,000 terms)
  h->codes = std::move(code);
  struct Slice {
    void **dst;
    const void *src;
    size_t bytes, off;
  };
  std::vector<Slice> slices;
  size_t total = 0;
  auto add = [&](auto *&dst, const auto &vec) {
    using E = typename std::remove_reference<decltype(vec)>::type::value_type;
    const size_t bytes = vec.size() * sizeof(E);
    slices.push_back({reinterpret_cast<void **>(&dst), vec.data(), bytes, total});
    total += (std::max<size_t>(bytes, sizeof(E)) + 255) & ~(size_t)255;
  };
  add(h->d_groups, h->groups);
  add(h->d_nodes, h->nodes);
  add(h->d_leaf_coef, h->leaf_coef);
  add(h->d_term_leaf, h->term_leaf);
  add(h->d_zmask, h->zmask);
  add(h->d_offdiag, h->offdiag);
  add(h->d_codes, h->codes);
  add(h->d_coeffs, h->coeffs);
  add(h->d_sumidx_shared, sumidx_shared);
  add(h->d_sumidx_word, sumidx_word);
  add(h->d_wordlist, wl);
  if (h->cut >= 0) {
    add(h->d_sl_groups, h->sl_groups);
    add(h->d_sl_nodes, h->sl_nodes);
    add(h->d_sr_groups, h->sr_groups);
    add(h->d_sr_nodes, h->sr_nodes);
    add(h->d_pairs, h->pairs);
    add(h->d_split_leaf_coef, h->split_leaf_coef);
    add(h->d_split_term_leaf, h->split_term_leaf);
    add(h->d_pl_off, h->pl_off);
    add(h->d_pr_off, h->pr_off);
    add(h->d_pr_idx, h->pr_idx);
    add(h->d_pair_sign, h->pair_sign);
  }
  {
    std::vector<unsigned char> image(total, 0);
    for (const Slice &sl : slices)
      if (sl.bytes) std::memcpy(image.data() + sl.off, sl.src, sl.bytes);
    CUDA_TRY(ctx, cudaMalloc(&h->d_arena, std::max<size_t>(total, 256)));
    for (const Slice &sl : slices) *sl.dst = h->d_arena + sl.off;
    CUDA_TRY(ctx, cudaMemcpy(h->d_arena, image.data(), total, cudaMemcpyHostToDevice));
  }
  const int id = ctx->next_handle++;
  ctx->hams[id] = std::move(h);
  *handle = id;
  return VQEMPS_OK;
}

// Batches of at least this many states evaluate energies with the per-term-cut
// plan (multicut_plan.inc); smaller ones with the single cut, so callers that
// evaluate a Hamiltonian a few states at a time never pay for the build.
constexpr int MC_MIN_BATCH = 32;

// Build and upload the per-term-cut plan once (one device allocation), then
// release its inputs.
static int ensure_multicut(vqemps_ctx *ctx, Hamiltonian *h) {
  if (!h->mc_pending) return VQEMPS_OK;
  h->mc_pending = false;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  build_multicut_plan(*h);
  std::vector<int32_t>().swap(h->mc_rslot);
  std::vector<int32_t>().swap(h->mc_sid_count);
  if (!h->mc_built) return VQEMPS_OK;
  struct Slice {
    void **dst;
    const void *src;
    size_t bytes, off;
  };
  std::vector<Slice> slices;
  size_t total = 0;
  auto add = [&](auto *&dst, const auto &vec) {
    using E = typename std::remove_reference<decltype(vec)>::type::value_type;
    const size_t bytes = vec.size() * sizeof(E);
    slices.push_back({reinterpret_cast<void **>(&dst), vec.data(), bytes, total});
    total += (std::max<size_t>(bytes, sizeof(E)) + 255) & ~(size_t)255;
  };
  add(h->d_mp_groups, h->mp_groups);
  add(h->d_mp_nodes, h->mp_nodes);
  add(h->d_ms_groups, h->ms_groups);
  add(h->d_ms_nodes, h->ms_nodes);
  add(h->d_mc_pairs, h->mc_pairs);
  add(h->d_mc_pair_sign, h->mc_pair_sign);
  add(h->d_mc_leaf_coef, h->mc_leaf_coef);
  add(h->d_mc_term_leaf, h->mc_term_leaf);
  std::vector<unsigned char> image(total, 0);
  for (const Slice &sl : slices)
    if (sl.bytes) std::memcpy(image.data() + sl.off, sl.src, sl.bytes);
  const cudaError_t e = cudaMalloc(&h->d_arena_mc, std::max<size_t>(total, 256));
  if (e != cudaSuccess) {
    h->mc_built = false;
    h->d_arena_mc = nullptr;
    return fail(ctx, VQEMPS_CUDA_ERROR, std::string("per-term-cut plan upload: ") + cudaGetErrorString(e));
  }
  for (const Slice &sl : slices) *sl.dst = h->d_arena_mc + sl.off;
  CUDA_TRY(ctx, cudaMemcpy(h->d_arena_mc, image.data(), total, cudaMemcpyHostToDevice));
  return VQEMPS_OK;
}

// The energy path's plan for this call (B states): sets h->mcut, which the leaf
// accessors and run_levels follow.
static int select_plan(vqemps_ctx *ctx, Hamiltonian *h, int B) {
  h->mcut = false;
  if (h->cut < 0 || B < MC_MIN_BATCH) return VQEMPS_OK;
  const int rc = ensure_multicut(ctx, h);
  if (rc) return rc;
  h->mcut = h->mc_built;
  return VQEMPS_OK;
}

extern "C" int vqemps_free_hamiltonian(vqemps_ctx *ctx, int handle) {
  if (!ctx) return VQEMPS_INVALID;
  cudaSetDevice(ctx->device);
  ctx->hams.erase(handle);
  return VQEMPS_OK;
}

// Work statistics of a plan (for benchmarks): flops of one evaluation of one state
// as executed, the survey-style count (16 Dl Dr (Dl + Dr) per trie node-site),
// node-sites, groups, leaves.
extern "C" int vqemps_plan_stats(const vqemps_ctx *ctx, int handle, double *stats) {
  if (!ctx || !stats) return VQEMPS_INVALID;
  auto it = ctx->hams.find(handle);
  if (it == ctx->hams.end()) return VQEMPS_INVALID;
  Hamiltonian &h = *it->second;
  // the plan of a large batch: the per-term-cut plan where it applies
  const int rc = ensure_multicut(const_cast<vqemps_ctx *>(ctx), &h);
  if (rc) return rc;
  const bool mc = h.mc_built;
  const bool split = h.cut >= 0;
  stats[0] = mc ? h.mc_flops : split ? h.split_flops : h.flops;
  stats[1] = h.flops_survey;
  stats[2] = mc ? (double)h.mc_node_sites : split ? (double)h.split_node_sites : (double)h.node_sites;
  stats[3] = mc ? (double)h.mc_groups_total
                : split ? (double)(h.sl_groups.size() + h.sr_groups.size()) : (double)h.groups.size();
  stats[4] = (double)(mc ? h.mc_nleaf : split ? h.split_nleaf : h.nleaf);
  stats[5] = mc ? (double)h.mc_max_slot : split ? (double)std::max(h.sl_max_slot, h.sr_max_slot) : (double)h.max_slot;
  stats[6] = (double)h.cut;
  stats[7] = h.flops;
  stats[8] = (double)h.node_sites;
  stats[9] = (double)(mc ? h.mc_npairs : h.npairs);
  return VQEMPS_OK;
}

// ---------------------------------------------------------------------------
// batched energy
// ---------------------------------------------------------------------------
static int ensure_state_ws(vqemps_ctx *ctx, int B) {
  const int n = ctx->n;
  if (B > 65535) return fail(ctx, VQEMPS_INVALID, "at most 65535 parameter sets per call");
  CUDA_TRY(ctx, ctx->sites.ensure((size_t)B * n * SITE_ELEMS));
  CUDA_TRY(ctx, ctx->bonds_ws.ensure((size_t)B * (n + 1)));
  CUDA_TRY(ctx, ctx->status.ensure((size_t)B));
  CUDA_TRY(ctx, ctx->right.ensure((size_t)B * (n + 1) * ENV_ELEMS));
  return VQEMPS_OK;
}

// Two-CTA gate chains halve the chain's critical path but double the CTAs: they
// pay while every state's pair of CTAs finds room next to the others (measured on
// B200 at 40 qubits: 1.3x faster at B <= 128, slower at B = 256), so by default
// they run while B is at most the SM count.
static bool use_pair_chain(const vqemps_ctx *ctx, int B) {
  // two 128-thread CTAs per state: up to 2 x SM count states stay resident at once
  return ctx->evolve_pair > 0 || (ctx->evolve_pair < 0 && B <= 2 * ctx->sm_count);
}

// Four CTAs per state (circuits of real gates) when the four-gate schedule is
// shorter than the two-gate one and all B clusters are resident at once (a second
// wave would double the chain's time); forced by mode 2.
static bool use_quad_chain(vqemps_ctx *ctx, int B) {
  if (!ctx->real_circuit || ctx->evolve_pair == 0 || ctx->evolve_pair == 1) return false;
  if (ctx->evolve_pair == 2) return true;
  if (ctx->qsteps >= ctx->psched.nsteps) return false;
  // measured on the 40-qubit benchmark circuit: four CTAs per state win while the
  // GPU holds at most about four CTAs per SM (B <= 128: 1.09 against 1.29 ms); with
  // more, the extra resident warps only wait at the CTA barriers (B = 256: 1.48
  // against 1.44 ms with two CTAs per state)
  if (B > ctx->sm_count) return false;
  if (ctx->quad_clusters < 0) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(4 * 8 * ctx->sm_count);
    cfg.blockDim = dim3(PAIR_THREADS);
    cfg.dynamicSmemBytes = EvolveSmemReal::bytes(ctx->n);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 4;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, (void *)evolve_quad_real_kernel, &cfg) != cudaSuccess) {
      cudaGetLastError();
      nc = 0;
    }
    ctx->quad_clusters = nc;
  }
  return B <= ctx->quad_clusters;
}

static int launch_evolve(vqemps_ctx *ctx, const double *theta_dev, int B, cudaStream_t st) {
  EvolveParams ep{};
  ep.gates = ctx->d_gates;
  ep.ngates = (int)ctx->gates.size();
  ep.mats = ctx->d_mats;
  ep.n = ctx->n;
  ep.P = ctx->P;
  ep.theta = theta_dev;
  ep.sites = ctx->sites.ptr;
  ep.bonds = ctx->bonds_ws.ptr;
  ep.status = ctx->status.ptr;
  ep.init0 = ctx->init0;
  ep.init1 = ctx->init1;
  ep.max_bond = ctx->max_bond;
  ep.abs_cut = ctx->abs_cut;
  ep.rel_cut = ctx->rel_cut;
  ctx->evolve_launches = 1;
  const bool quad = use_quad_chain(ctx, B);
  if (quad || use_pair_chain(ctx, B)) {
    // every two-site gate's pending one-site products, formed in parallel
    CUDA_TRY(ctx, ctx->upend.ensure((size_t)B * std::max(ep.ngates, 1) * 8));
    ep.gate_q = ctx->d_gate_q;
    ep.qlist = ctx->d_qlist;
    if (ep.ngates > 0) {
      pending_kernel<<<dim3((ep.ngates + 127) / 128, B), 128, 0, st>>>(ep, ctx->upend.ptr);
      CUDA_TRY(ctx, cudaGetLastError());
      ctx->evolve_launches = 2;
    }
    ep.upend = ctx->upend.ptr;
  }
  if (quad) {
    ep.sched = ctx->d_qsched;
    ep.nsteps = ctx->qsteps;
    ep.gate_q = ctx->d_gate_q;
    ep.qlist = ctx->d_qlist;
    ep.tail_off = ctx->d_tail_off;
    evolve_quad_real_kernel<<<4 * B, PAIR_THREADS, EvolveSmemReal::bytes(ctx->n), st>>>(ep);
  } else if (use_pair_chain(ctx, B)) {
    ep.sched = ctx->d_sched;
    ep.nsteps = ctx->psched.nsteps;
    ep.gate_q = ctx->d_gate_q;
    ep.qlist = ctx->d_qlist;
    ep.tail_off = ctx->d_tail_off;
    if (ctx->real_circuit)
      evolve_pair_real_kernel<<<2 * B, PAIR_THREADS, EvolveSmem::bytes(ctx->n), st>>>(ep);
    else
      evolve_pair_kernel<<<2 * B, PAIR_THREADS, EvolveSmem::bytes(ctx->n), st>>>(ep);
  } else {
    if (ctx->real_circuit)
      evolve_real_kernel<<<B, EVOLVE_THREADS, EvolveSmem::bytes(ctx->n), st>>>(ep);
    else
      evolve_kernel<<<B, EVOLVE_THREADS, EvolveSmem::bytes(ctx->n), st>>>(ep);
  }
  CUDA_TRY(ctx, cudaGetLastError());
  return VQEMPS_OK;
}

// Identity right environments (and the sampler's branch matrices when branch
// is non-null); writes the norm into the identity leaf of h when given.
static int launch_right(vqemps_ctx *ctx, Hamiltonian *h, int B, cudaStream_t st, cplx *branch) {
  const int nleaf = h ? std::max(h->e_nleaf(), 1) : 0;
  if (h) CUDA_TRY(ctx, ctx->leafval.ensure((size_t)B * nleaf));
  if (ctx->real_circuit) {
    // real arithmetic, and the real copies the real-arithmetic levels stage: R,
    // the site panels and, for a split plan, the transposed panels
    const bool panels = h != nullptr, panels_t = h != nullptr && h->cut >= 0;
    CUDA_TRY(ctx, ctx->right_real.ensure((size_t)B * (ctx->n + 1) * ENV_ELEMS));
    if (panels) CUDA_TRY(ctx, ctx->panels.ensure((size_t)B * ctx->n * RL_PANEL));
    if (panels_t) CUDA_TRY(ctx, ctx->panels_t.ensure((size_t)B * ctx->n * RL_PANEL));
    right_env_real_kernel<<<B, RIGHT_THREADS, 0, st>>>(ctx->sites.ptr, ctx->n, ctx->right.ptr, branch,
                                                      ctx->status.ptr, h ? ctx->leafval.ptr : nullptr, nleaf,
                                                      h ? h->e_identity_leaf() : -1, ctx->right_real.ptr,
                                                      panels ? ctx->panels.ptr : nullptr,
                                                      panels_t ? ctx->panels_t.ptr : nullptr);
    ctx->right_real_fresh = true;
    ctx->panels_fresh = panels;
    ctx->panels_t_fresh = panels_t;
  } else {
    right_env_kernel<<<B, RIGHT_THREADS, 0, st>>>(ctx->sites.ptr, ctx->n, ctx->right.ptr, branch,
                                                 ctx->status.ptr, h ? ctx->leafval.ptr : nullptr,
                                                 nleaf, h ? h->e_identity_leaf() : -1);
    ctx->right_real_fresh = ctx->panels_fresh = ctx->panels_t_fresh = false;
  }
  CUDA_TRY(ctx, cudaGetLastError());
  return VQEMPS_OK;
}

// Level kernel variants: the autotuner times each on the caller's workload.

// Parents per warp of the prefetch DMMA kernels: 8 on wide levels, 4 on
// middling ones, fewer while the whole batch would give less than two waves of
// resident CTAs (three per SM), so that small batches keep every SM busy. The
// values do not depend on it: each parent is computed the same way by any warp.
static int mpf_parents_per_warp(int ng, int B, int sms) {
  int gpw = ng >= 32 * MPF_WARPS ? 8 : (ng >= 4 * MPF_WARPS ? 4 : 1);
  while (gpw > 1 && (long long)((ng + MPF_WARPS * gpw - 1) / (MPF_WARPS * gpw)) * B < 6LL * sms) gpw >>= 1;
  return gpw;
}

static void launch_level_variant(int variant, const LevelParams &lp, int ng, int B, int sms, cudaStream_t st) {
  switch (variant) {
    case LV_MMA4:
      level_mma_kernel<4><<<dim3((ng + 3) / 4, B), 4 * 32, sizeof(LevelMmaSmem<4>), st>>>(lp);
      break;
    case LV_MMA8:
      level_mma_kernel<8><<<dim3((ng + 7) / 8, B), 8 * 32, sizeof(LevelMmaSmem<8>), st>>>(lp);
      break;
    case LV_PF4: {
      // about four parents per warp, never fewer than one CTA per state
      const int gpw = ng >= 4 * PF_WARPS ? 4 : 1;
      const int ctas = (ng + PF_WARPS * gpw - 1) / (PF_WARPS * gpw);
      level_pf_kernel<<<dim3(ctas, B), PF_WARPS * 32, sizeof(LevelPfSmem), st>>>(lp, gpw);
      break;
    }
    case LV_MMAPF4: {
      const int gpw = mpf_parents_per_warp(ng, B, sms);
      const int ctas = (ng + MPF_WARPS * gpw - 1) / (MPF_WARPS * gpw);
      level_mma_pf_kernel<<<dim3(ctas, B), MPF_WARPS * 32, sizeof(LevelMmaPfSmem), st>>>(lp, gpw);
      break;
    }
    case LV_MMA3PF4: {
      const int gpw = mpf_parents_per_warp(ng, B, sms);
      const int ctas = (ng + MPF_WARPS * gpw - 1) / (MPF_WARPS * gpw);
      level_mma3_pf_kernel<<<dim3(ctas, B), MPF_WARPS * 32, sizeof(LevelMmaPfSmem), st>>>(lp, gpw);
      break;
    }
    case LV_REALPF4: {
      const int gpw = mpf_parents_per_warp(ng, B, sms);
      const int ctas = (ng + RL_WARPS * gpw - 1) / (RL_WARPS * gpw);
      level_real_pf_kernel<<<dim3(ctas, B), RL_WARPS * 32, sizeof(LevelRealSmem), st>>>(lp, gpw);
      break;
    }
    default:
      level_kernel<<<dim3((ng + LEVEL_WARPS - 1) / LEVEL_WARPS, B), LEVEL_WARPS * 32, sizeof(LevelSmem), st>>>(lp);
  }
}

// All trie levels of one evaluation with a given variant (needs launch_right first).
// Inputs of the real-arithmetic levels that launch_right did not write: real
// site panels (and transposed ones for suffix levels) and the real parts of R.
static int prepare_real_inputs(vqemps_ctx *ctx, int B, bool transposed, cudaStream_t st) {
  const int n = ctx->n;
  int &nl = ctx->level_launches;
  CUDA_TRY(ctx, ctx->panels.ensure((size_t)B * n * RL_PANEL));
  CUDA_TRY(ctx, ctx->right_real.ensure((size_t)B * (n + 1) * ENV_ELEMS));
  if (!(ctx->right_real_fresh && ctx->panels_fresh)) {
    real_panels_kernel<<<dim3(n, B), 256, 0, st>>>(ctx->sites.ptr, n, 0, ctx->panels.ptr);
    CUDA_TRY(ctx, cudaGetLastError());
    ++nl;
  }
  if (transposed && !(ctx->right_real_fresh && ctx->panels_t_fresh)) {
    CUDA_TRY(ctx, ctx->panels_t.ensure((size_t)B * n * RL_PANEL));
    real_panels_kernel<<<dim3(n, B), 256, 0, st>>>(ctx->sites.ptr, n, 1, ctx->panels_t.ptr);
    CUDA_TRY(ctx, cudaGetLastError());
    ++nl;
  }
  if (!ctx->right_real_fresh) {       // launch_right wrote only the complex environments
    const size_t rcount = (size_t)B * (n + 1) * ENV_ELEMS;
    real_parts_kernel<<<(unsigned)std::min<size_t>((rcount + 255) / 256, 4096), 256, 0, st>>>(
        ctx->right.ptr, rcount, ctx->right_real.ptr);
    CUDA_TRY(ctx, cudaGetLastError());
    ++nl;
  }
  return VQEMPS_OK;
}

// Fork the split evaluation's suffix half onto the second stream: returns the
// stream to launch it on (joined back by join_suffix before the pair closures).
static int fork_suffix(vqemps_ctx *ctx, cudaStream_t st, cudaStream_t *sst) {
  if (!ctx->aux) {
    CUDA_TRY(ctx, cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking));
    CUDA_TRY(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
    CUDA_TRY(ctx, cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  }
  CUDA_TRY(ctx, cudaEventRecord(ctx->ev_fork, st));
  CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->aux, ctx->ev_fork, 0));
  *sst = ctx->aux;
  return VQEMPS_OK;
}
static int join_suffix(vqemps_ctx *ctx, cudaStream_t st, cudaStream_t sst) {
  CUDA_TRY(ctx, cudaEventRecord(ctx->ev_join, sst));
  CUDA_TRY(ctx, cudaStreamWaitEvent(st, ctx->ev_join, 0));
  return VQEMPS_OK;
}

// All trie levels of one evaluation with the per-term-cut plan (h.mcut): the
// suffix levels (second stream) and the prefix levels write their environments
// into per-level regions of mflat_s / mflat_p, then the pair closures.
static int run_levels_mcut(vqemps_ctx *ctx, Hamiltonian &h, int B, cudaStream_t st, int variant) {
  const int n = ctx->n;
  const int nleaf = std::max(h.e_nleaf(), 1);
  const bool real = variant == LV_REALPF4;
  int &nl = ctx->level_launches;
  nl = 0;
  if (real) {
    const int rc = prepare_real_inputs(ctx, B, true, st);
    if (rc) return rc;
  }
  // a region's first element: real environments are ENV_ELEMS doubles, complex ones ENV_ELEMS cplx
  const size_t unit = real ? 1 : 2;
  auto region = [&](DevBuf<cplx> &f, int base) {
    return reinterpret_cast<cplx *>(reinterpret_cast<double *>(f.ptr) + (size_t)B * base * ENV_ELEMS * unit);
  };
  cudaStream_t sst = st;
  {
    const int rc = fork_suffix(ctx, st, &sst);
    if (rc) return rc;
  }
  if (!real) {
    transpose_sites_kernel<<<dim3(n, B), 256, 0, sst>>>(ctx->sites.ptr, n, ctx->sites_t.ptr);
    CUDA_TRY(ctx, cudaGetLastError());
    ++nl;
  }
  for (int s = n - 1; s >= h.ms_low; --s) {
    const int ng = h.ms_group_off[s + 1] - h.ms_group_off[s];
    if (ng == 0) continue;                        // sites beyond every suffix path
    LevelParams lp{};
    lp.sites = ctx->sites_t.ptr;
    lp.right = ctx->right.ptr;
    lp.env_prev = region(ctx->mflat_s, s + 1 < n ? h.ms_base[s + 1] : 0);
    lp.env_cur = region(ctx->mflat_s, h.ms_base[s]);
    lp.groups = h.d_ms_groups + h.ms_group_off[s];
    lp.nodes = h.d_ms_nodes + h.ms_node_off[s];
    lp.leafval = ctx->leafval.ptr;
    lp.ngroups = ng;
    lp.nslot_prev = s + 1 < n ? h.ms_stride[s + 1] : 1;
    lp.nslot_cur = h.ms_stride[s];
    lp.nleaf_total = nleaf;
    lp.n = n;
    lp.s = s;
    lp.suffix = 1;
    lp.flip = s & 1;
    lp.panels = ctx->panels_t.ptr;
    lp.right_real = ctx->right_real.ptr;
    lp.status = ctx->status.ptr;
    launch_level_variant(variant == LV_MMA3PF4 || variant == LV_REALPF4 ? variant : LV_MMAPF4, lp, ng, B,
                         ctx->sm_count, sst);
    CUDA_TRY(ctx, cudaGetLastError());
    ++nl;
  }
  for (int s = 0; s < h.mp_levels; ++s) {
    const int ng = h.mp_group_off[s + 1] - h.mp_group_off[s];
    if (ng == 0) continue;
    LevelParams lp{};
    lp.sites = ctx->sites.ptr;
    lp.right = ctx->right.ptr;
    lp.env_prev = region(ctx->mflat_p, s > 0 ? h.mp_base[s - 1] : 0);
    lp.env_cur = region(ctx->mflat_p, h.mp_base[s]);
    lp.groups = h.d_mp_groups + h.mp_group_off[s];
    lp.nodes = h.d_mp_nodes + h.mp_node_off[s];
    lp.leafval = ctx->leafval.ptr;
    lp.ngroups = ng;
    lp.nslot_prev = s > 0 ? h.mp_stride[s - 1] : 1;
    lp.nslot_cur = h.mp_stride[s];
    lp.nleaf_total = nleaf;
    lp.n = n;
    lp.s = s;
    lp.flip = s & 1;
    lp.panels = ctx->panels.ptr;
    lp.right_real = ctx->right_real.ptr;
    lp.status = ctx->status.ptr;
    launch_level_variant(variant, lp, ng, B, ctx->sm_count, st);
    CUDA_TRY(ctx, cudaGetLastError());
    ++nl;
  }
  {
    const int rc = join_suffix(ctx, st, sst);
    if (rc) return rc;
  }
  if (h.mc_npairs > 0) {
    const dim3 grid((h.mc_npairs + COMBINE_WARPS - 1) / COMBINE_WARPS, B);
    if (real)
      pair_combine_real_kernel<<<grid, COMBINE_WARPS * 32, 0, st>>>(
          reinterpret_cast<const double *>(ctx->mflat_p.ptr), reinterpret_cast<const double *>(ctx->mflat_s.ptr),
          h.d_mc_pairs, h.d_mc_pair_sign, h.mc_npairs, ctx->status.ptr, ctx->leafval.ptr, nleaf);
    else
      pair_combine_kernel<<<grid, COMBINE_WARPS * 32, 0, st>>>(ctx->mflat_p.ptr, ctx->mflat_s.ptr, h.d_mc_pairs,
                                                               h.mc_npairs, ctx->status.ptr, ctx->leafval.ptr,
                                                               nleaf);
    CUDA_TRY(ctx, cudaGetLastError());
    ++nl;
  }
  return VQEMPS_OK;
}

static int run_levels(vqemps_ctx *ctx, Hamiltonian &h, int B, cudaStream_t st, int variant) {
  if (variant == LV_REALPF4 && !ctx->real_circuit)
    return fail(ctx, VQEMPS_INVALID, "the real-arithmetic level kernels need a circuit of real gates");
  if (h.mcut) return run_levels_mcut(ctx, h, B, st, variant);
  const int n = ctx->n;
  const int nleaf = std::max(h.e_nleaf(), 1);
  const bool split = h.cut >= 0;
  const int top = split ? h.cut : n;                // prefix levels run on sites 0 .. top - 1
  const bool real = variant == LV_REALPF4;
  int &nl = ctx->level_launches;
  nl = 0;
  if (real) {
    const int rc2 = prepare_real_inputs(ctx, B, split, st);
    if (rc2) return rc2;
  }
  // the suffix half (stream sst) and the prefix half are independent until the
  // pair closures: fork the suffix half onto the second stream
  cudaStream_t sst = st;
  if (split) {
    const int rc2 = fork_suffix(ctx, st, &sst);
    if (rc2) return rc2;
  }
  if (split) {
    // suffix levels n-1 .. cut on transposed site tensors, starting from R_{l+1}
    if (!real) {
      transpose_sites_kernel<<<dim3(n, B), 256, 0, sst>>>(ctx->sites.ptr, n, ctx->sites_t.ptr);
      CUDA_TRY(ctx, cudaGetLastError());
      ++nl;
    }
    cplx *renv[2] = {ctx->env2.ptr, ctx->env3.ptr};
    for (int s = n - 1; s >= h.cut; --s) {
      const int ng = h.sr_group_off[s + 1] - h.sr_group_off[s];
      if (ng == 0) continue;                        // sites beyond every term's last
      LevelParams lp{};
      lp.sites = ctx->sites_t.ptr;
      lp.right = ctx->right.ptr;
      lp.env_prev = renv[(s + 1) & 1];
      lp.env_cur = renv[s & 1];
      lp.groups = h.d_sr_groups + h.sr_group_off[s];
      lp.nodes = h.d_sr_nodes + h.sr_node_off[s];
      lp.leafval = ctx->leafval.ptr;
      lp.ngroups = ng;
      lp.nslot_prev = s + 1 < n ? std::max(h.sr_nslot[s + 1], 1) : 1;
      lp.nslot_cur = std::max(h.sr_nslot[s], 1);
      lp.nleaf_total = nleaf;
      lp.n = n;
      lp.s = s;
      lp.suffix = 1;
      lp.flip = s & 1;
      lp.panels = ctx->panels_t.ptr;
      lp.right_real = ctx->right_real.ptr;
      lp.status = ctx->status.ptr;
      launch_level_variant(variant == LV_MMA3PF4 || variant == LV_REALPF4 ? variant : LV_MMAPF4, lp, ng, B,
                           ctx->sm_count, sst);
      CUDA_TRY(ctx, cudaGetLastError());
      ++nl;
    }
  }
  cplx *envs[2] = {ctx->env0.ptr, ctx->env1.ptr};
  for (int s = 0; s < top; ++s) {
    const int ng = h.group_off[s + 1] - h.group_off[s];
    if (ng == 0) break;
    LevelParams lp{};
    lp.sites = ctx->sites.ptr;
    lp.right = ctx->right.ptr;
    lp.env_prev = envs[(s + 1) & 1];
    lp.env_cur = envs[s & 1];
    lp.groups = (split ? h.d_sl_groups : h.d_groups) + h.group_off[s];
    lp.nodes = (split ? h.d_sl_nodes : h.d_nodes) + h.node_off[s];
    lp.leafval = ctx->leafval.ptr;
    lp.ngroups = ng;
    lp.nslot_prev = s > 0 ? std::max(h.nslot[s - 1], 1) : 1;
    lp.nslot_cur = std::max(h.nslot[s], 1);
    lp.nleaf_total = nleaf;
    lp.n = n;
    lp.s = s;
    lp.flip = s & 1;
    lp.panels = ctx->panels.ptr;
    lp.right_real = ctx->right_real.ptr;
    lp.status = ctx->status.ptr;
    launch_level_variant(variant, lp, ng, B, ctx->sm_count, st);
    CUDA_TRY(ctx, cudaGetLastError());
    ++nl;
  }
  if (split) {   // join the suffix half
    const int rc2 = join_suffix(ctx, st, sst);
    if (rc2) return rc2;
  }
  if (split && h.npairs > 0) {
    const dim3 grid((h.npairs + COMBINE_WARPS - 1) / COMBINE_WARPS, B);
    cplx *left = envs[(h.cut - 1) & 1], *right = (h.cut & 1) ? ctx->env3.ptr : ctx->env2.ptr;
    if (variant == LV_REALPF4)
      split_combine_real_kernel<<<grid, COMBINE_WARPS * 32, 0, st>>>(
          reinterpret_cast<const double *>(left), std::max(h.nslot[h.cut - 1], 1),
          reinterpret_cast<const double *>(right), std::max(h.sr_nslot[h.cut], 1), h.d_pairs, h.d_pair_sign,
          h.npairs, ctx->status.ptr, ctx->leafval.ptr, nleaf);
    else
      split_combine_kernel<<<grid, COMBINE_WARPS * 32, 0, st>>>(
          left, std::max(h.nslot[h.cut - 1], 1), right, std::max(h.sr_nslot[h.cut], 1), h.d_pairs, h.npairs,
          ctx->status.ptr, ctx->leafval.ptr, nleaf);
    CUDA_TRY(ctx, cudaGetLastError());
    ++nl;
  }
  return VQEMPS_OK;
}

static int batch_bucket(int B) {
  int k = 0;
  while ((1 << k) < B) ++k;
  return k;
}

// Variant for (plan, batch size): forced, cached, or measured now. Tuning
// times every variant once on the prepared states (CUDA events, synchronising
// the stream once per plan and batch-size bucket) and keeps the fastest.
// A plan's size class for the autotuner: its batch-size bucket, split or prefix
// evaluation, and the power-of-two bucket of its node-sites per state. Which
// kernel is fastest follows from these (how many groups a level launch has per
// state, and how many states share it), so a decision made on one plan is reused
// for the next plan of the same class instead of timing every variant again --
// the usual case when a solver loads one Hamiltonian after another.
static int shape_key(const Hamiltonian &h, int B) {
  const long long sites = h.cut >= 0 ? h.split_node_sites : h.node_sites;
  int lg = 0;
  while ((1LL << lg) < std::max(sites, 1LL)) ++lg;
  return (batch_bucket(B) * 2 + (h.cut >= 0 ? 1 : 0)) * 64 + lg;
}

static int pick_variant(vqemps_ctx *ctx, Hamiltonian &h, int B, cudaStream_t st, int *variant) {
  if (ctx->forced_variant >= 0) { *variant = ctx->forced_variant; return VQEMPS_OK; }
  const int key = batch_bucket(B);
  auto it = h.tuned.find(key);
  if (it != h.tuned.end()) { *variant = it->second; return VQEMPS_OK; }
  const int skey = shape_key(h, B);
  auto sit = ctx->tuned_by_shape.find(skey);
  if (sit != ctx->tuned_by_shape.end()) {
    h.tuned[key] = sit->second;
    *variant = sit->second;
    return VQEMPS_OK;
  }
  // the two timing events are destroyed on every exit path
  struct Events {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Events() {
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    }
  } ev;
  CUDA_TRY(ctx, cudaEventCreate(&ev.e0));
  CUDA_TRY(ctx, cudaEventCreate(&ev.e1));
  int best = LV_SIMT4;
  float best_ms = 1e30f;
  for (int v = 0; v < LV_COUNT; ++v) {
    if (v == LV_REALPF4 && !ctx->real_circuit) continue;   // complex amplitudes
    int rc = run_levels(ctx, h, B, st, v);      // warm
    if (rc) return rc;
    CUDA_TRY(ctx, cudaEventRecord(ev.e0, st));
    rc = run_levels(ctx, h, B, st, v);
    if (rc) return rc;
    CUDA_TRY(ctx, cudaEventRecord(ev.e1, st));
    CUDA_TRY(ctx, cudaEventSynchronize(ev.e1));
    float ms = 0.f;
    CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ev.e0, ev.e1));
    if (ms < best_ms) { best_ms = ms; best = v; }
  }
  h.tuned[key] = best;
  ctx->tuned_by_shape[skey] = best;
  *variant = best;
  return VQEMPS_OK;
}

// Trie levels and the energy reduction on the prepared states (needs launch_right first).
static int launch_levels(vqemps_ctx *ctx, Hamiltonian &h, int B, cudaStream_t st,
                         double *energies_dev, double *per_term_dev) {
  const int nleaf = std::max(h.e_nleaf(), 1);
  CUDA_TRY(ctx, ctx->leafval.ensure((size_t)B * nleaf));
  if (h.mcut) {
    // every level keeps its environments (complex size; the real levels use half)
    CUDA_TRY(ctx, ctx->mflat_p.ensure((size_t)B * h.mp_slots * ENV_ELEMS));
    CUDA_TRY(ctx, ctx->mflat_s.ensure((size_t)B * h.ms_slots * ENV_ELEMS));
    CUDA_TRY(ctx, ctx->sites_t.ensure((size_t)B * ctx->n * SITE_ELEMS));
  } else {
    const size_t pre_slots = h.cut >= 0 ? h.sl_max_slot : h.max_slot;
    CUDA_TRY(ctx, ctx->env0.ensure((size_t)B * pre_slots * ENV_ELEMS));
    CUDA_TRY(ctx, ctx->env1.ensure((size_t)B * pre_slots * ENV_ELEMS));
    if (h.cut >= 0) {
      CUDA_TRY(ctx, ctx->env2.ensure((size_t)B * h.sr_max_slot * ENV_ELEMS));
      CUDA_TRY(ctx, ctx->env3.ensure((size_t)B * h.sr_max_slot * ENV_ELEMS));
      CUDA_TRY(ctx, ctx->sites_t.ensure((size_t)B * ctx->n * SITE_ELEMS));
    }
  }
  int variant = LV_SIMT4;
  int rc = pick_variant(ctx, h, B, st, &variant);
  if (rc) return rc;
  rc = run_levels(ctx, h, B, st, variant);
  if (rc) return rc;
  reduce_kernel<<<B, REDUCE_THREADS, 0, st>>>(ctx->leafval.ptr, h.e_leaf_coef(), h.e_nleaf(),
                                             h.e_term_leaf(), h.T, ctx->status.ptr, energies_dev,
                                             per_term_dev);
  CUDA_TRY(ctx, cudaGetLastError());
  return VQEMPS_OK;
}

// Gate chain: 1 two-CTA clusters on an as-soon-as-possible schedule, 0 one CTA
// in program order, -1 (default) two-CTA clusters while B <= the SM count.
// Same states bit for bit.
extern "C" int vqemps_set_evolve_mode(vqemps_ctx *ctx, int mode) {
  if (!ctx || mode < -1 || mode > 2) return VQEMPS_INVALID;
  ctx->evolve_pair = mode;
  return VQEMPS_OK;
}

// Split evaluation of Hamiltonians loaded afterwards: -1 when it saves work
// (default), 0 never, 1 always (at the best cut).
extern "C" int vqemps_set_split_mode(vqemps_ctx *ctx, int mode) {
  if (!ctx || mode < -1 || mode > 1) return VQEMPS_INVALID;
  ctx->split_mode = mode;
  return VQEMPS_OK;
}

// Force a level kernel variant (0 SIMT, 1 DMMA x4 warps, 2 DMMA x8 warps) or
// restore autotuning (-1); query the variant a plan uses for a batch size.
extern "C" int vqemps_set_level_variant(vqemps_ctx *ctx, int variant) {
  if (!ctx || variant < -1 || variant >= LV_COUNT) return VQEMPS_INVALID;
  ctx->forced_variant = variant;
  return VQEMPS_OK;
}

static Hamiltonian *find_ham(vqemps_ctx *ctx, int handle) {
  auto it = ctx->hams.find(handle);
  return it == ctx->hams.end() ? nullptr : it->second.get();
}

extern "C" int vqemps_level_variant(vqemps_ctx *ctx, int handle, int B, int *variant) {
  if (!ctx || !variant) return VQEMPS_INVALID;
  Hamiltonian *h = find_ham(ctx, handle);
  if (!h) return VQEMPS_INVALID;
  if (ctx->forced_variant >= 0) { *variant = ctx->forced_variant; return VQEMPS_OK; }
  auto it = h->tuned.find(batch_bucket(B));
  *variant = it == h->tuned.end() ? -1 : it->second;
  return VQEMPS_OK;
}

extern "C" int vqemps_energy_batch(vqemps_ctx *ctx, int handle, const double *theta_dev, int B,
                                   double *energies_dev, double *per_term_dev, void *stream) {
  if (!ctx) return VQEMPS_INVALID;
  if (!ctx->have_circuit) return fail(ctx, VQEMPS_INVALID, "no circuit");
  Hamiltonian *h = find_ham(ctx, handle);
  if (!h) return fail(ctx, VQEMPS_INVALID, "unknown Hamiltonian handle");
  if (B < 1 || (!theta_dev && ctx->P > 0) || !energies_dev)
    return fail(ctx, VQEMPS_INVALID, "bad batch arguments");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = as_stream(stream);
  int rc = select_plan(ctx, h, B);
  if (rc) return rc;
  rc = ensure_state_ws(ctx, B);
  if (rc) return rc;
  rc = launch_evolve(ctx, theta_dev, B, st);
  if (rc) return rc;
  rc = launch_right(ctx, h, B, st, nullptr);
  if (rc) return rc;
  rc = launch_levels(ctx, *h, B, st, energies_dev, per_term_dev);
  if (rc) return rc;
  ctx->last_B = B;
  return VQEMPS_OK;
}

// Phase timing of one batched energy call: ms[0] state preparation, ms[1]
// right environments, ms[2] all trie levels, ms[3] reduction; *launches = kernels
// launched. Records CUDA events on the stream and synchronises it.
extern "C" int vqemps_profile_energy(vqemps_ctx *ctx, int handle, const double *theta_dev, int B,
                                     double *ms, int *launches, void *stream) {
  if (!ctx || !ms || !launches) return VQEMPS_INVALID;
  Hamiltonian *h = find_ham(ctx, handle);
  if (!h || B < 1) return fail(ctx, VQEMPS_INVALID, "bad profile arguments");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = as_stream(stream);
  int rc = select_plan(ctx, h, B);
  if (rc) return rc;
  rc = ensure_state_ws(ctx, B);
  if (rc) return rc;
  CUDA_TRY(ctx, ctx->energy_stage.ensure((size_t)B));
  cudaEvent_t ev[5];
  for (auto &e : ev) CUDA_TRY(ctx, cudaEventCreate(&e));
  CUDA_TRY(ctx, cudaEventRecord(ev[0], st));
  rc = launch_evolve(ctx, theta_dev, B, st);
  if (rc) return rc;
  CUDA_TRY(ctx, cudaEventRecord(ev[1], st));
  rc = launch_right(ctx, h, B, st, nullptr);
  if (rc) return rc;
  CUDA_TRY(ctx, cudaEventRecord(ev[2], st));
  // levels and reduction are launched by launch_levels; time them apart by a
  // second call of the reduction alone
  rc = launch_levels(ctx, *h, B, st, ctx->energy_stage.ptr, nullptr);
  if (rc) return rc;
  CUDA_TRY(ctx, cudaEventRecord(ev[3], st));
  reduce_kernel<<<B, REDUCE_THREADS, 0, st>>>(ctx->leafval.ptr, h->e_leaf_coef(), h->e_nleaf(),
                                             h->e_term_leaf(), h->T, ctx->status.ptr, ctx->energy_stage.ptr,
                                             nullptr);
  CUDA_TRY(ctx, cudaGetLastError());
  CUDA_TRY(ctx, cudaEventRecord(ev[4], st));
  CUDA_TRY(ctx, cudaEventSynchronize(ev[4]));
  float t[4];
  for (int i = 0; i < 4; ++i) CUDA_TRY(ctx, cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]));
  ms[0] = t[0];
  ms[1] = t[1];
  ms[3] = t[3];
  ms[2] = t[2] - t[3];   // launch_levels includes one reduction
  *launches = ctx->evolve_launches + 1 + ctx->level_launches + 1;   // gate chain, right env, levels, reduction
  for (auto &e : ev) cudaEventDestroy(e);
  ctx->last_B = B;
  return VQEMPS_OK;
}

extern "C" int vqemps_batch_status(vqemps_ctx *ctx, int32_t *status, int B, void *stream) {
  if (!ctx || !status || B < 1 || B > ctx->last_B) return VQEMPS_INVALID;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = as_stream(stream);
  CUDA_TRY(ctx, cudaMemcpyAsync(status, ctx->status.ptr, sizeof(int32_t) * B, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  int first = VQEMPS_OK;
  for (int b = 0; b < B; ++b)
    if (status[b] != 0) { first = status[b]; break; }
  if (first == VQEMPS_INSUFFICIENT_BOND)
    ctx->err = "CUDAQ_MPS_MAX_BOND=" + std::to_string(ctx->max_bond) +
               " is insufficient for zero-cutoff simulation: resolved singular values would be discarded";
  else if (first == VQEMPS_NONFINITE_SVD)
    ctx->err = "Direct MPS SVD failed or produced nonfinite singular values";
  else if (first == VQEMPS_TIMEOUT)
    ctx->err = "a bounded device wait gave up (bulk copy or barrier did not complete)";
  return first;
}

extern "C" int vqemps_energy_batch_host(vqemps_ctx *ctx, int handle, const double *theta, int B,
                                        double *energies, double *per_term, void *stream) {
  if (!ctx) return VQEMPS_INVALID;
  if (!ctx->have_circuit) return fail(ctx, VQEMPS_INVALID, "no circuit");
  Hamiltonian *h = find_ham(ctx, handle);
  if (!h) return fail(ctx, VQEMPS_INVALID, "unknown Hamiltonian handle");
  if (B < 1 || (!theta && ctx->P > 0) || !energies) return fail(ctx, VQEMPS_INVALID, "bad batch arguments");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = as_stream(stream);
  CUDA_TRY(ctx, ctx->theta_stage.ensure((size_t)B * std::max(ctx->P, 1)));
  CUDA_TRY(ctx, ctx->energy_stage.ensure((size_t)B));
  if (per_term) CUDA_TRY(ctx, ctx->per_term_stage.ensure((size_t)B * std::max(h->T, 1)));
  if (ctx->P > 0)
    CUDA_TRY(ctx, cudaMemcpyAsync(ctx->theta_stage.ptr, theta, sizeof(double) * B * ctx->P,
                                  cudaMemcpyHostToDevice, st));
  int rc = vqemps_energy_batch(ctx, handle, ctx->theta_stage.ptr, B, ctx->energy_stage.ptr,
                               per_term ? ctx->per_term_stage.ptr : nullptr, stream);
  if (rc) return rc;
  CUDA_TRY(ctx, cudaMemcpyAsync(energies, ctx->energy_stage.ptr, sizeof(double) * B,
                                cudaMemcpyDeviceToHost, st));
  if (per_term)
    CUDA_TRY(ctx, cudaMemcpyAsync(per_term, ctx->per_term_stage.ptr, sizeof(double) * B * h->T,
                                  cudaMemcpyDeviceToHost, st));
  std::vector<int32_t> status(B);
  return vqemps_batch_status(ctx, status.data(), B, stream);
}

extern "C" int vqemps_copy_sites(vqemps_ctx *ctx, int b, double *sites_host, void *stream) {
  if (!ctx || !sites_host || b < 0 || b >= ctx->last_B) return VQEMPS_INVALID;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = as_stream(stream);
  CUDA_TRY(ctx, cudaMemcpyAsync(sites_host, ctx->sites.ptr + (size_t)b * ctx->n * SITE_ELEMS,
                                sizeof(cplx) * ctx->n * SITE_ELEMS, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return VQEMPS_OK;
}

#include "engine_sample.inc"
#include "engine_grad.inc"
#include "engine_parts.inc"
#include "noalloc.cu"
