/*
 * vqemps.h -- C ABI of the B200 matrix-product-state engine for the VQE hot path.
 *
 * Plain pointers and sizes only. Device pointers (suffix _dev) are owned by the
 * caller (for example torch tensors' data_ptr()); the engine owns only its
 * workspaces. Every call returns a status code (vqemps_status). Calls taking a
 * stream are stream-ordered and do not synchronise the device, except where a
 * comment says so.
 *
 * Each entry point replaces a part of the reference's CUDA-Q NVQIR plugin
 * (test/backend/source/simulator_mps_dist.cu, class SimulatorMPSDist) or of its
 * Python reverse-mode gradient (test/tools/reverse_mps.py); paths are relative to
 * the hp-cyber/Graph-VQE project root.
 */
#ifndef VQEMPS_ABI_H
#define VQEMPS_ABI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The reference throws std::runtime_error or calls exit(1):
 * dist_svd.cuh:22-27 (CUDA/library errors), :277-279 (insufficient bond),
 * :280-281 (failed or nonfinite SVD), sharded_mps.cuh:643-645 (invalid Pauli),
 * simulator_mps_dist.cu:235-237,412-415 (too few qubits, unsupported gate). */
enum vqemps_status {
  VQEMPS_OK = 0,
  VQEMPS_INSUFFICIENT_BOND = 1, /* zero-cutoff rank guard fired (reference devInfo rank -2) */
  VQEMPS_NONFINITE_SVD = 2,     /* nonfinite singular values / no convergence (rank -1)  */
  VQEMPS_INVALID = 3,           /* bad argument, gate, Pauli character or size           */
  VQEMPS_CUDA_ERROR = 4,        /* CUDA runtime error                                    */
  VQEMPS_TIMEOUT = 5            /* a bounded device wait gave up                          */
};

/* Gate kinds of vqemps_op. Rotations follow CUDA-Q: RX/RY/RZ(t) = exp(-i t P / 2). */
enum vqemps_gate {
  VQEMPS_RX = 0, VQEMPS_RY = 1, VQEMPS_RZ = 2,
  VQEMPS_H = 3, VQEMPS_X = 4, VQEMPS_Y = 5, VQEMPS_Z = 6, VQEMPS_S = 7, VQEMPS_SDG = 8,
  VQEMPS_CX = 9,    /* q0 = control, q1 = target                                         */
  VQEMPS_U1 = 10,   /* 2x2 row-major matrix from the matrix table, on q0                 */
  VQEMPS_U2 = 11,   /* 4x4 row-major [(I*2+J)*4+(i*2+j)] on (q0 -> I, q1 -> J)            */
  VQEMPS_SWAP = 12
};

/* Initial product state of every qubit (reverse_mps.py:41-43). */
enum vqemps_initial { VQEMPS_INIT_ZERO = 0, VQEMPS_INIT_ONE = 1, VQEMPS_INIT_PLUS = 2, VQEMPS_INIT_MINUS = 3 };

/* Random number generator of the sampler. SPLITMIX reproduces the reference's
 * per-(seed, site, shot) hash draw (sharded_mps.cuh:147-170); PHILOX is
 * Philox4x32-10 with counter (shot, site, 0, 0) and key (seed lo, seed hi). */
enum vqemps_rng { VQEMPS_RNG_SPLITMIX = 0, VQEMPS_RNG_PHILOX = 1 };

/* One circuit operation. A GateApplicationTask of the plugin
 * (simulator_mps_dist.cu:1392-1406) is {name, matrix, controls, targets,
 * parameters}; here it is {kind, qubits, parameter index or constant angle,
 * matrix-table index}. */
typedef struct vqemps_op {
  int32_t kind;    /* vqemps_gate                                          */
  int32_t q0;      /* target (1q), control (CX), first qubit (U2, SWAP)    */
  int32_t q1;      /* target (CX), second qubit (U2, SWAP), else -1        */
  int32_t param;   /* rotation angle = theta[param] * scale, or -1          */
  double angle;    /* rotation angle when param < 0; scale when param >= 0 */
  int32_t matrix;  /* index into the matrix table (U1: 4, U2: 16 complex)  */
  int32_t pad;
} vqemps_op;

typedef struct vqemps_ctx vqemps_ctx;

/* Create an engine on a CUDA device. Replaces SimulatorMPSDist::ensureEngine's
 * configuration (simulator_mps_dist.cu:363-366: CUDAQ_MPS_MAX_BOND /
 * _ABS_CUTOFF / _RELATIVE_CUTOFF) and the thread-local handle pool
 * (sharded_mps.cuh:276-305). max_bond <= 16 (the engine's padded bond). */
int vqemps_create(int device, int max_bond, double abs_cut, double rel_cut, vqemps_ctx **out);

/* Release all device memory of the engine (ShardedMPS::~ShardedMPS,
 * sharded_mps.cuh:413-427; AnalyticWorkspace::release, analytic_batch.cuh:44-52). */
int vqemps_destroy(vqemps_ctx *ctx);

/* Message of the last failing call on this context (never NULL). */
const char *vqemps_last_error(const vqemps_ctx *ctx);

/* Load a circuit: replaces addQubitsToState + the applyGate sequence of one
 * kernel execution (simulator_mps_dist.cu:1371-1406, 376-416). Qubit q maps to
 * MPS site q when site_order == 0, and to site n-1-q when site_order == 1 (the
 * plugin's msb map conv(q) = n-1-q, simulator_mps_dist.cu:387). Non-adjacent
 * two-qubit gates are routed by SWAPs as in ShardedMPS::applyTwoQubit
 * (sharded_mps.cuh:565-572). matrices: nmatrices complex numbers as (re, im)
 * pairs. Returns VQEMPS_INVALID for n < 2 (simulator_mps_dist.cu:235-237) or an
 * unsupported gate (:412-415). */
int vqemps_set_circuit(vqemps_ctx *ctx, int n, const vqemps_op *ops, int nops,
                       const double *matrices, int nmatrices, int initial, int site_order);

/* Number of circuit parameters (largest param index + 1) and bond dimensions
 * (n + 1 entries) that the zero-cutoff SVD keeps, the allocation bound of
 * graph_resources.allocation_bound (test/tools/graph_resources.py:12-32). */
int vqemps_num_params(const vqemps_ctx *ctx, int *params);
int vqemps_bond_dims(const vqemps_ctx *ctx, int *dims);

/* Load a Pauli sum: words is T rows of n characters over {I,X,Y,Z}, indexed by
 * QUBIT (row t, column q); coeffs are the real coefficients. The shared-prefix
 * plan is built and uploaded once per Hamiltonian (the reference rebuilds its
 * key-cached plan and re-uploads it on every call: sharded_mps.cuh:627-672).
 * Replaces buildPauliTermData (simulator_mps_dist.cu:571-583). */
int vqemps_set_hamiltonian(vqemps_ctx *ctx, const char *words, const double *coeffs, int T,
                           int *handle);
int vqemps_free_hamiltonian(vqemps_ctx *ctx, int handle);

/* Analytic energies of B parameter sets: E[b] = sum_k c_k Re<psi_b|P_k|psi_b>.
 * Replaces observe() with shots = -1 (simulator_mps_dist.cu:1434-1485) and
 * expectPauliShared (sharded_mps.cuh:614-687) for B states in one call.
 * theta_dev: B x P doubles; energies_dev: B doubles; per_term_dev: B x T doubles
 * of <P_k> (the ExecutionResult per term id, simulator_mps_dist.cu:1467-1481) or
 * NULL. Stream-ordered; per-state failures are reported by vqemps_batch_status. */
int vqemps_energy_batch(vqemps_ctx *ctx, int handle, const double *theta_dev, int B,
                        double *energies_dev, double *per_term_dev, void *stream);

/* Same as vqemps_energy_batch with HOST buffers: copies theta in and energies
 * (and per_term when non-NULL) out on the stream, then synchronises the stream
 * and returns the first per-state failure as the status. */
int vqemps_energy_batch_host(vqemps_ctx *ctx, int handle, const double *theta, int B,
                             double *energies, double *per_term, void *stream);

/* Per-state status of the last batched call (synchronises the stream). */
int vqemps_batch_status(vqemps_ctx *ctx, int32_t *status, int B, void *stream);

/* Energy and gradient dE/dtheta of B parameter sets through the exact
 * bond-doubling MPS (no SVD), the quantity of ReverseMPS.value_gradient
 * (reverse_mps.py:84-99). grad_dev: B x P doubles. Requires a circuit whose
 * two-qubit gates are adjacent CX (the ReverseMPS/register restriction,
 * reverse_mps.py:12-25). */
int vqemps_energy_grad_batch(vqemps_ctx *ctx, int handle, const double *theta_dev, int B,
                             double *energies_dev, double *grad_dev, void *stream);

/* Environment checkpointing of the gradient (no reference counterpart; the
 * reference bounds memory by 128-term chunks, reverse_mps.py:91-96): the forward
 * sweep keeps every `every`-th level, the backward sweep recomputes the rest one
 * segment at a time. Default 8; 1 keeps every level (no recomputation). */
int vqemps_set_grad_checkpoint(vqemps_ctx *ctx, int every);
/* Gradient level kernels (no reference counterpart): 0 = SIMT FMA kernels,
 * 1 = FP64 DMMA tensor-core kernels, 2 = DMMA with Gauss's three-product complex
 * multiply in the forward levels (default); for a circuit of real gates, 2 runs
 * the real-gate DMMA kernels (one real product per complex one; energies and
 * angle gradients equal variant 1's bit for bit). All give the same values to
 * rounding; VQEMPS_GRAD_VARIANT (simt, dmma, dmma3) selects one at creation. */
int vqemps_set_grad_variant(vqemps_ctx *ctx, int variant);

/* Perfect sampling of B states: shots bitstrings each, bit q of shot s of state
 * b in packed_dev[(b * shots + s) * W + q / 64] >> (q % 64), W = ceil(n / 64),
 * QUBIT order, n <= 256. Replaces sample() without noise
 * (simulator_mps_dist.cu:1587-1613) and sampleBitsGpu (sharded_mps.cuh:814-902).
 * seed is the evaluation seed of state 0 (the plugin's sampleSeed++ value); state
 * b uses seed + b. With VQEMPS_RNG_SPLITMIX the draw seed is
 * hbatchSeedForShotShard(seed + b, 0) (simulator_mps_dist.cu:596-608), so with
 * site_order 1 the shots are the plugin's. */
int vqemps_sample(vqemps_ctx *ctx, const double *theta_dev, int B, int shots, uint64_t seed,
                  int rng, uint64_t *packed_dev, void *stream);

/* Shot-estimated energies. Replaces observe() with finite shots
 * (simulator_mps_dist.cu:1487-1515). Words with X or Y are evaluated
 * analytically in both modes (evaluateHbatchTermBatch, simulator_mps_dist.cu:661-700).
 * mode VQEMPS_SHOTS_SHARED: every I/Z word is estimated from one shared sample
 *   set per state (runSharedDiagonalShotBatch, :1157-1171; sampleZExpectationsGpu,
 *   sharded_mps.cuh:906-935).
 * mode VQEMPS_SHOTS_PLUGIN: the plugin's rule -- shared when every word is I/Z,
 *   otherwise an independent stream per non-identity I/Z word
 *   (sampleZExpectationsIndependentGpu, sharded_mps.cuh:942-982).
 * seed is the evaluation seed of state 0 (state b uses seed + b).
 * per_term_dev (B x T) or NULL. */
enum vqemps_shot_mode { VQEMPS_SHOTS_SHARED = 0, VQEMPS_SHOTS_PLUGIN = 1 };
int vqemps_sampled_energy(vqemps_ctx *ctx, int handle, const double *theta_dev, int B, int shots,
                          uint64_t seed, int rng, int mode, double *energies_dev,
                          double *per_term_dev, void *stream);

/* Level-kernel selection (no reference counterpart). The trie levels have six
 * implementations: 0 FP64 CUDA-core (SIMT) kernel, 1 FP64 tensor-core (DMMA)
 * kernel with 4 warps per CTA, 2 DMMA with 8 warps per CTA, 3 SIMT with
 * persistent warps that prefetch the next parent environment (cp.async),
 * 4 DMMA with the same prefetching pipeline, 5 the same with Gauss's
 * three-product complex multiply. By default the
 * engine times each once per plan and batch-size bucket (powers of two) on the
 * first call and keeps the fastest (that first call synchronises its stream);
 * vqemps_set_level_variant forces one (-1 restores tuning);
 * vqemps_level_variant reports the one in use (-1: not tuned yet). The
 * environment variable VQEMPS_LEVEL_VARIANT (simt, dmma4, dmma8, simt_pf,
 * dmma_pf, dmma3_pf or 0-5), read by vqemps_create, forces one for every context. */
int vqemps_set_level_variant(vqemps_ctx *ctx, int variant);
int vqemps_level_variant(vqemps_ctx *ctx, int handle, int B, int *variant);

/* Benchmark support (no reference counterpart): phase times of one batched
 * energy call -- ms[0] state preparation, ms[1] right environments, ms[2] trie
 * levels, ms[3] energy reduction -- and the number of kernels one call launches.
 * Synchronises the stream. */
int vqemps_profile_energy(vqemps_ctx *ctx, int handle, const double *theta_dev, int B, double *ms,
                          int *launches, void *stream);

/* Work statistics of a loaded Pauli sum, per state and evaluation (stats[10]):
 * [0] FP64 flops of the energy path as executed, [1] the survey count
 * 16 Dl Dr (Dl + Dr) per node-site of the prefix trie, [2] node-sites as
 * executed, [3] parent groups, [4] leaves, [5] largest environment slot count of
 * a level, [6] cut site of the single-cut split evaluation (-1: prefix trie
 * only; the energy path then closes each word at its own cut when that needs
 * fewer node-sites), [7] / [8] flops / node-sites of the prefix trie alone,
 * [9] prefix/suffix pair closures. */
int vqemps_plan_stats(const vqemps_ctx *ctx, int handle, double *stats);

/* Split evaluation (no reference counterpart; the reference walks prefix tries
 * only, sharded_mps.cuh:614-687): a Pauli sum loaded afterwards is evaluated as
 * a prefix trie up to a cut site plus a suffix trie from the cut, each word
 * closed by one dot product of its prefix and suffix environments when that
 * needs fewer node-sites. mode -1 (default): when it saves at least 15 % of the
 * node-sites; 0: never; 1: always, at the best cut. Same values to rounding. */
int vqemps_set_split_mode(vqemps_ctx *ctx, int mode);

/* Gate chain (no reference counterpart; the reference applies gates one by one,
 * simulator_mps_dist.cu:1392-1406): 1 runs each state on a cluster of two CTAs
 * that apply two-site gates on disjoint site pairs concurrently, on an
 * as-soon-as-possible schedule built with the circuit; 2 (circuits of real gates;
 * others as 1) on a cluster of four CTAs, up to four gates per step; 0 runs one
 * CTA per state in program order; -1 (default) uses 2 for a circuit of real gates
 * while all clusters of four fit the GPU at once and the four-gate schedule is
 * shorter, else 1 while the batch has at most twice as many states as the GPU has
 * SMs, else 0. All give the same states bit for bit. */
int vqemps_set_evolve_mode(vqemps_ctx *ctx, int mode);

/* Copy the site tensors of state b of the last batched call to the host:
 * n * 16 * 2 * 16 complex (re, im) pairs, site s at offset s * 1024 doubles,
 * element (l, p, r) at ((l * 2 + p) * 16 + r), zero padded beyond the bond dims.
 * Used to check the prepared state against the oracle (synchronises). */
int vqemps_copy_sites(vqemps_ctx *ctx, int b, double *sites_host, void *stream);

/* Partition sets: K independent circuits of uneven width, parameter count and
 * Hamiltonian evaluated in one batch. Replaces the plain partition warm start's
 * sequential local solves, one observe() per energy and partition
 * (test/sources/independent-vqe/Qiskit_VQE/independent_vqe.py:276-290 ->
 * test/tools/independent_campaign.py:15-63 _minimize_model). Partition k has
 * ns[k] qubits, ops[op_off[k] .. op_off[k+1]) (matrix indices relative to
 * matrices + 2 * matrix_off[k], matrix_off may be NULL), and the Pauli sum of
 * rows term_off[k] .. term_off[k+1] of coeffs, whose words are packed one
 * partition after another, each ns[k] characters wide (qubit order, as
 * vqemps_set_hamiltonian). Every partition compiles exactly as a one-circuit
 * engine would; initial state and site order are shared. */
int vqemps_set_partitions(vqemps_ctx *ctx, int K, const int32_t *ns, const vqemps_op *ops,
                          const int32_t *op_off, const double *matrices, const int32_t *matrix_off,
                          const char *words, const int64_t *term_off, const double *coeffs,
                          int initial, int site_order, int *handle);
int vqemps_free_partitions(vqemps_ctx *ctx, int handle);
/* info[6]: K, widest partition n_max, theta row stride P_max, per-term row
 * stride T_max, 64-bit words per shot W, trie levels; params[K] (may be NULL):
 * parameters of each partition; flops (may be NULL): FP64 flops of one
 * evaluation of every partition. */
int vqemps_partition_info(vqemps_ctx *ctx, int handle, int32_t *info, int32_t *params, double *flops);
/* Allocation bounds of partition k (ns[k] + 1 entries). */
int vqemps_partition_bond_dims(vqemps_ctx *ctx, int handle, int k, int *dims);
/* Analytic energies of copies parameter sets of every partition: state
 * b = k * copies + c; theta_dev (K * copies) x P_max (partition k reads the
 * first P_k entries of its rows), energies_dev K * copies, per_term_dev
 * (optional) (K * copies) x T_max. Status per state: vqemps_batch_status. */
int vqemps_partition_energy(vqemps_ctx *ctx, int handle, const double *theta_dev, int copies,
                            double *energies_dev, double *per_term_dev, void *stream);
/* Bitstrings of every state: packed_dev (K * copies) x shots x W, bit q of a
 * shot is qubit q of its partition; state b uses evaluation seed seed + b, as
 * vqemps_sample. */
int vqemps_partition_sample(vqemps_ctx *ctx, int handle, const double *theta_dev, int copies, int shots,
                            uint64_t seed, int rng, uint64_t *packed_dev, void *stream);
/* Shot-estimated energies from one shared sample set per state (I/Z words from
 * the shots, X/Y words analytic: VQEMPS_SHOTS_SHARED semantics). packed_dev
 * (optional) receives the shots as vqemps_partition_sample writes them. */
int vqemps_partition_sampled_energy(vqemps_ctx *ctx, int handle, const double *theta_dev, int copies,
                                    int shots, uint64_t seed, int rng, double *energies_dev,
                                    double *per_term_dev, uint64_t *packed_dev, void *stream);

/* Allocation-free analytic energy of ONE parameter set. No counterpart in the
 * reference: it exists for callers that must not allocate device memory while
 * they run -- for example a simulator plugin hosted inside a runtime that owns
 * all device memory through its own pool, or an operator under a fixed memory
 * budget -- because vqemps_energy_batch grows its workspaces with cudaMalloc.
 * All intermediate data live in one static device array of 22 MiB per GPU,
 * held until the process exits. Limits: <= 64 qubits, <= 2560 environments kept
 * on one site, <= 16384 distinct term endings (VQEMPS_INVALID beyond them).
 * Calls share that array: calls that overlap on the GPU race and must be
 * serialised by the caller. The first call on a device looks the array up
 * (make it before any stream capture); the address is tied to the CUDA context
 * current at that call, and after a device reset the next call looks it up
 * again (it too must come before any capture). The caller's current device is
 * the same after the call as before it. theta_dev: P doubles; energy_dev: 1
 * double (NaN if the state failed); per_term_dev: T doubles or NULL;
 * status_dev: 1 int32 (vqemps_status of the state) or NULL. */
int vqemps_energy_noalloc(vqemps_ctx *ctx, int handle, const double *theta_dev, double *energy_dev,
                          double *per_term_dev, int32_t *status_dev, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* VQEMPS_ABI_H */
