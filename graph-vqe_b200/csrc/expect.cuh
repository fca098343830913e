// Pauli-sum expectations by shared-prefix left sweeps.
//
// Reference algorithm (test/backend/source):
//   expectPauliShared ......... sharded_mps.cuh:614-687 (sorted words, prefix trie)
//   analyticLeft/Right/Gather . analytic_batch.cuh:4-36  (E' = A^H P E A per node)
//   k_rightStage/k_rightFinish  sharded_mps.cuh:61-90    (identity right environments)
// and the same contraction in test/tools/reverse_mps.py:59-82 (energy_chunk).
//
// B200 design. The trie is built once per Hamiltonian over ALL terms (the
// reference chunks it into <= 128-term pieces and re-uploads it per call) and
// every path stops at its term's last non-identity site: there the value is
// closed against the identity right environment R_{s+1} of the state, which is
// computed once per state. Work is level-synchronous (one launch per site) and
// batched over B parameter sets. A warp owns one trie parent: it computes
// S_i = E_parent A_i once for all of its children, then one product per Pauli
// class present among the children: {I, Z} share t_i = A_i^H S_i
// (I = t_0 + t_1, Z = t_0 - t_1) and {X, Y} share u_01 = A_0^H S_1 and
// u_10 = A_1^H S_0 (X = u_01 + u_10, Y = -i u_01 + i u_10). The site tile is
// staged once per CTA in shared memory; environments are FP64 16 x 16.
#pragma once
#include "common.cuh"

namespace vqemps {

struct DevGroup {   // one trie parent with its children at the current level
  int32_t parent_slot;   // env slot of the parent in the previous level (-1: root)
  int32_t child_begin;   // first child node (index within the level)
  int32_t nchild;
  int32_t classes;       // bit 0: an I or Z child, bit 1: an X or Y child, bit 2: the
                         // parent's phase (Y count) is odd (prefix and single-cut plans)
};

struct DevNode {    // one trie node
  int32_t code;          // 0 I, 1 X, 2 Y, 3 Z
  int32_t env_slot;      // slot in this level's env buffer, -1 if no descendants
  int32_t leaf;          // leaf id if a term ends here, else -1
  int32_t phase;         // number of Y codes on the node's path, mod 4: for a state
                         // with real amplitudes the node's environment is i^phase
                         // times a real matrix (the real-arithmetic levels use it)
};

// ---------------------------------------------------------------------------
// Identity right environments: R_n = 1,
// R_s[b,b'] = sum_{i,c,c'} conj(A_s[b,i,c]) R_{s+1}[c,c'] A_s[b',i,c'].
// One CTA per state; R stored for s = 0..n (n+1 tiles of 16x16). When branch is
// non-null the two physical-index parts M_0, M_1 of every R_s are stored too
// (the sampler's branch probabilities).
// ---------------------------------------------------------------------------
constexpr int RIGHT_THREADS = 256;

__device__ __forceinline__ void right_env_body(const cplx *__restrict__ sb, int n, cplx *__restrict__ rb,
                                               cplx *__restrict__ mbase, bool ok, double *leafslot) {
  // site tile rows padded to 33 elements: the first contraction's 16 rows of a
  // half-warp then fall on distinct banks
  constexpr int AS = 2 * CHI + 1;
  __shared__ cplx A[CHI * AS];
  __shared__ cplx R[ENV_ELEMS];
  __shared__ cplx T[2 * ENV_ELEMS];
  const int tid = threadIdx.x;
  R[tid] = cmake(tid == 0 ? 1.0 : 0.0, 0.0);
  rb[(size_t)n * ENV_ELEMS + tid] = R[tid];
  for (int s = n - 1; s >= 0; --s) {
    for (int e = tid; e < SITE_ELEMS; e += RIGHT_THREADS) A[(e >> 5) * AS + (e & 31)] = sb[(size_t)s * SITE_ELEMS + e];
    __syncthreads();
    // T_i[c, b'] = sum_c' R[c,c'] A[b',i,c']
    {
      const int c = tid >> 4, bp = tid & 15;
      cplx t0 = cmake(0, 0), t1 = cmake(0, 0);
      for (int cp = 0; cp < CHI; ++cp) {
        const cplx r = R[c * CHI + cp];
        cfma(t0, r, A[bp * AS + cp]);
        cfma(t1, r, A[bp * AS + CHI + cp]);
      }
      T[c * CHI + bp] = t0;
      T[ENV_ELEMS + c * CHI + bp] = t1;
    }
    __syncthreads();
    // R_s[bb, b'] = sum_i M_i[bb, b'],  M_i[bb, b'] = sum_c conj(A[bb,i,c]) T_i[c,b']
    {
      const int bb = tid >> 4, bp = tid & 15;
      cplx m0 = cmake(0, 0), m1 = cmake(0, 0);
      for (int c = 0; c < CHI; ++c) {
        cfma_conj(m0, A[bb * AS + c], T[c * CHI + bp]);
        cfma_conj(m1, A[bb * AS + CHI + c], T[ENV_ELEMS + c * CHI + bp]);
      }
      const cplx acc = cadd(m0, m1);
      R[tid] = acc;
      rb[(size_t)s * ENV_ELEMS + tid] = acc;
      if (mbase != nullptr) {
        cplx *mb = mbase + (size_t)s * 2 * ENV_ELEMS;
        mb[tid] = m0;
        mb[ENV_ELEMS + tid] = m1;
      }
    }
    __syncthreads();
  }
  if (leafslot != nullptr && tid == 0) *leafslot = ok ? R[0].x : 0.0;
}

__global__ void __launch_bounds__(RIGHT_THREADS)
right_env_kernel(const cplx *__restrict__ sites, int n, cplx *__restrict__ right,
                 cplx *__restrict__ branch, const int32_t *__restrict__ status,
                 double *__restrict__ leafval, int nleaf_total, int identity_leaf) {
  const int b = blockIdx.x;
  right_env_body(sites + (size_t)b * n * SITE_ELEMS, n, right + (size_t)b * (n + 1) * ENV_ELEMS,
                 branch ? branch + (size_t)b * n * 2 * ENV_ELEMS : nullptr, status[b] == 0,
                 identity_leaf >= 0 ? leafval + (size_t)b * nleaf_total + identity_leaf : nullptr);
}

// Partition sets: state b belongs to partition st_part[b] of width part_n[]
// (sites / right / branch strides follow the widest partition, n_max) and
// identity leaf part_idleaf[] (-1 if none).
__global__ void __launch_bounds__(RIGHT_THREADS)
right_env_multi_kernel(const cplx *__restrict__ sites, int n_max, const int32_t *__restrict__ st_part,
                       const int32_t *__restrict__ part_n, const int32_t *__restrict__ part_idleaf,
                       cplx *__restrict__ right, cplx *__restrict__ branch, const int32_t *__restrict__ status,
                       double *__restrict__ leafval, int leaf_stride) {
  const int b = blockIdx.x;
  const int k = st_part[b];
  const int idl = part_idleaf[k];
  right_env_body(sites + (size_t)b * n_max * SITE_ELEMS, part_n[k], right + (size_t)b * (n_max + 1) * ENV_ELEMS,
                 branch ? branch + (size_t)b * n_max * 2 * ENV_ELEMS : nullptr, status[b] == 0,
                 (leafval && idl >= 0) ? leafval + (size_t)b * leaf_stride + idl : nullptr);
}

// ---------------------------------------------------------------------------
// One trie level for B states.
// ---------------------------------------------------------------------------
constexpr int LEVEL_WARPS = 4;

struct LevelParams {
  const cplx *sites;        // B x n x SITE_ELEMS
  const cplx *right;        // B x (n+1) x ENV_ELEMS
  const cplx *env_prev;     // B x nslot_prev x ENV_ELEMS (unused at s = 0)
  cplx *env_cur;            // B x nslot_cur x ENV_ELEMS
  const DevGroup *groups;   // this level's groups
  const DevNode *nodes;     // this level's nodes
  double *leafval;          // B x nleaf_total
  int ngroups, nslot_prev, nslot_cur, nleaf_total;
  int n, s;
  // Uneven batches: work items (state, first group, group count) of this level,
  // three ints each, one per CTA (null: state = blockIdx.y, all groups).
  const int32_t *work;
  // Suffix levels of the split evaluation (prefix-pipeline kernels only): sites
  // holds transposed site tensors and a group without a parent slot starts from
  // the identity right environment R_{s+1} instead of the vacuum.
  int suffix;
  // Real-arithmetic levels: real padded site panels [B][n][CHI * 36] doubles
  // (transposed ones for suffix levels), real parts of the identity right
  // environments [B][n + 1][ENV_ELEMS], and the per-state status words (a
  // bounded device wait that gives up writes ST_TIMEOUT there).
  const double *panels;
  const double *right_real;
  int32_t *status;
  // Nonzero: CTA row blockIdx.y works on state gridDim.y - 1 - blockIdx.y
  // (real-arithmetic levels). Consecutive levels alternate, so a level first
  // reads the parents its predecessor wrote last, while they are still in L2.
  int flip;
};

struct LevelSmem {
  cplx A[SITE_ELEMS];
  cplx W[LEVEL_WARPS][2 * ENV_ELEMS];   // per warp: parent E (first 4 KiB), then S_0 | S_1
};

// Lane layout (conflict-free shared-memory access): a quarter-warp (8 lanes with
// equal lane >> 3) always reads 8 consecutive complex numbers of one row
// (128 bytes) or one broadcast address.
//   first half:  rows 4*(lane>>3) .. +3 of S, columns (lane&7) + 8c, c = 0..3,
//                of the 32-column panel [S_0 | S_1]
//   second half: rows 4*(lane>>3) .. +3 of E', columns (lane&7) + 8c, c = 0..1
__global__ void __launch_bounds__(LEVEL_WARPS * 32, 4)
level_kernel(LevelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LevelSmem &sm = *reinterpret_cast<LevelSmem *>(smem_raw);
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
  for (int e = threadIdx.x; e < SITE_ELEMS; e += LEVEL_WARPS * 32) sm.A[e] = ag[e];
  __syncthreads();
  const int gidx = blockIdx.x * LEVEL_WARPS + warp;
  if (gidx >= p.ngroups) return;
  const DevGroup grp = p.groups[gidx];
  cplx *E = sm.W[warp];
  cplx *S = sm.W[warp];
  const cplx *A = sm.A;
  const int rq = lane >> 3, cq = lane & 7;

  // parent environment
  if (grp.parent_slot < 0) {
    for (int e = lane; e < ENV_ELEMS; e += 32) E[e] = cmake(e == 0 ? 1.0 : 0.0, 0.0);
  } else {
    const cplx *src = p.env_prev + ((size_t)b * p.nslot_prev + grp.parent_slot) * ENV_ELEMS;
    for (int e = lane; e < ENV_ELEMS; e += 32) E[e] = src[e];
  }
  __syncwarp();

  // ---- S_i[a, c] = sum_a' E[a, a'] A[a', i, c]
  {
    cplx acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[r][c] = cmake(0, 0);
#pragma unroll 2
    for (int k = 0; k < CHI; ++k) {
      cplx e[4], a[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) e[r] = E[(rq * 4 + r) * CHI + k];
#pragma unroll
      for (int c = 0; c < 4; ++c) a[c] = A[k * 2 * CHI + cq + 8 * c];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) cfma(acc[r][c], e[r], a[c]);
    }
    __syncwarp();            // all lanes are done reading E before S overwrites it
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c)  // panel column cq + 8c = i * 16 + c'
        S[(c >> 1) * ENV_ELEMS + (rq * 4 + r) * CHI + cq + 8 * (c & 1)] = acc[r][c];
  }
  __syncwarp();

  // ---- second half
  const cplx *R = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
  for (int cls = 0; cls < 2; ++cls) {
    if (!(grp.classes & (1 << cls))) continue;
    cplx t0[4][2], t1[4][2];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 2; ++c) { t0[r][c] = cmake(0, 0); t1[r][c] = cmake(0, 0); }
    // cls 0: t_i = A_i^H S_i ; cls 1: t0 = A_0^H S_1 (u01), t1 = A_1^H S_0 (u10)
    const int s0 = cls == 0 ? 0 : 1;
    const int s1 = cls == 0 ? 1 : 0;
#pragma unroll 2
    for (int a = 0; a < CHI; ++a) {
      cplx sv0[2], sv1[2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        sv0[c] = S[s0 * ENV_ELEMS + a * CHI + cq + 8 * c];
        sv1[c] = S[s1 * ENV_ELEMS + a * CHI + cq + 8 * c];
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const cplx av0 = A[(a * 2 + 0) * CHI + rq * 4 + r];
        const cplx av1 = A[(a * 2 + 1) * CHI + rq * 4 + r];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          cfma_conj(t0[r][c], av0, sv0[c]);
          cfma_conj(t1[r][c], av1, sv1[c]);
        }
      }
    }
    for (int ci = 0; ci < grp.nchild; ++ci) {
      const DevNode node = p.nodes[grp.child_begin + ci];
      const bool iz = (node.code == 0 || node.code == 3);
      if (iz != (cls == 0)) continue;
      cplx out[4][2];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          if (node.code == 0 || node.code == 1) out[r][c] = cadd(t0[r][c], t1[r][c]);
          else if (node.code == 3) out[r][c] = csub(t0[r][c], t1[r][c]);
          else {  // Y: -i u01 + i u10
            const cplx d = csub(t1[r][c], t0[r][c]);
            out[r][c] = cmake(-d.y, d.x);
          }
        }
      if (node.env_slot >= 0) {
        cplx *dst = p.env_cur + ((size_t)b * p.nslot_cur + node.env_slot) * ENV_ELEMS;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 2; ++c) dst[(rq * 4 + r) * CHI + cq + 8 * c] = out[r][c];
      }
      if (node.leaf >= 0) {
        double v = 0.0;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const cplx rv = R[(rq * 4 + r) * CHI + cq + 8 * c];
            v += out[r][c].x * rv.x - out[r][c].y * rv.y;
          }
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) p.leafval[(size_t)b * p.nleaf_total + node.leaf] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Prefetching variant: persistent warps walk several parents each. A warp owns a
// 4 KiB parent slot and an 8 KiB S panel; as soon as the first half of a parent
// is done the next parent's environment is copied into the slot with cp.async
// (16 bytes per lane per instruction), overlapping the second half. The CTA
// stages R_{s+1} next to the site tile. Same arithmetic and lane layout as
// level_kernel.
// ---------------------------------------------------------------------------
constexpr int PF_WARPS = 4;

struct LevelPfSmem {
  cplx A[SITE_ELEMS];
  cplx R[ENV_ELEMS];
  cplx E[PF_WARPS][ENV_ELEMS];          // per warp: parent environment slot
  cplx S[PF_WARPS][2 * ENV_ELEMS];      // per warp: S_0 | S_1
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Stage the parent environment of group g into E (cp.async, or the root identity).
__device__ __forceinline__ void stage_parent(const LevelParams &p, int b, int g, cplx *E, int lane) {
  const DevGroup grp = p.groups[g];
  if (grp.parent_slot < 0) {
    for (int e = lane; e < ENV_ELEMS; e += 32) E[e] = cmake(e == 0 ? 1.0 : 0.0, 0.0);
  } else {
    const cplx *src = p.env_prev + ((size_t)b * p.nslot_prev + grp.parent_slot) * ENV_ELEMS;
    for (int e = lane; e < ENV_ELEMS; e += 32) cp_async16(E + e, src + e);
  }
}

__global__ void __launch_bounds__(PF_WARPS * 32, 3)
level_pf_kernel(LevelParams p, int groups_per_warp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LevelPfSmem &sm = *reinterpret_cast<LevelPfSmem *>(smem_raw);
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {
    const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
    const cplx *rg = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
    for (int e = threadIdx.x; e < SITE_ELEMS; e += PF_WARPS * 32) sm.A[e] = ag[e];
    for (int e = threadIdx.x; e < ENV_ELEMS; e += PF_WARPS * 32) sm.R[e] = rg[e];
  }
  __syncthreads();
  const cplx *A = sm.A;
  const cplx *R = sm.R;
  const int rq = lane >> 3, cq = lane & 7;
  // this warp's parents: first, first + stride, ... (at most groups_per_warp)
  const int stride = gridDim.x * PF_WARPS;
  const int first = blockIdx.x * PF_WARPS + warp;
  int count = 0;
  if (first < p.ngroups) count = min(groups_per_warp, (p.ngroups - first + stride - 1) / stride);
  if (count == 0) return;
  cplx *E = sm.E[warp];
  cplx *S = sm.S[warp];
  stage_parent(p, b, first, E, lane);
  cp_async_commit();
  for (int k = 0; k < count; ++k) {
    const int gidx = first + k * stride;
    cp_async_wait<0>();
    __syncwarp();
    const DevGroup grp = p.groups[gidx];
    {
      cplx acc[4][4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = cmake(0, 0);
#pragma unroll 1
      for (int kk = 0; kk < CHI; ++kk) {
        cplx e[4], a[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) e[r] = E[(rq * 4 + r) * CHI + kk];
#pragma unroll
        for (int c = 0; c < 4; ++c) a[c] = A[kk * 2 * CHI + cq + 8 * c];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) cfma(acc[r][c], e[r], a[c]);
      }
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c)
          S[(c >> 1) * ENV_ELEMS + (rq * 4 + r) * CHI + cq + 8 * (c & 1)] = acc[r][c];
    }
    __syncwarp();   // E is dead and S is complete: prefetch the next parent
    if (k + 1 < count) stage_parent(p, b, gidx + stride, E, lane);
    cp_async_commit();
    for (int cls = 0; cls < 2; ++cls) {
      if (!(grp.classes & (1 << cls))) continue;
      cplx t0[4][2], t1[4][2];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c) { t0[r][c] = cmake(0, 0); t1[r][c] = cmake(0, 0); }
      const int s0 = cls == 0 ? 0 : 1;
      const int s1 = cls == 0 ? 1 : 0;
#pragma unroll 1
      for (int a = 0; a < CHI; ++a) {
        cplx sv0[2], sv1[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          sv0[c] = S[s0 * ENV_ELEMS + a * CHI + cq + 8 * c];
          sv1[c] = S[s1 * ENV_ELEMS + a * CHI + cq + 8 * c];
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const cplx av0 = A[(a * 2 + 0) * CHI + rq * 4 + r];
          const cplx av1 = A[(a * 2 + 1) * CHI + rq * 4 + r];
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            cfma_conj(t0[r][c], av0, sv0[c]);
            cfma_conj(t1[r][c], av1, sv1[c]);
          }
        }
      }
      for (int ci = 0; ci < grp.nchild; ++ci) {
        const DevNode node = p.nodes[grp.child_begin + ci];
        const bool iz = (node.code == 0 || node.code == 3);
        if (iz != (cls == 0)) continue;
        cplx out[4][2];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            if (node.code == 0 || node.code == 1) out[r][c] = cadd(t0[r][c], t1[r][c]);
            else if (node.code == 3) out[r][c] = csub(t0[r][c], t1[r][c]);
            else { const cplx d = csub(t1[r][c], t0[r][c]); out[r][c] = cmake(-d.y, d.x); }
          }
        if (node.env_slot >= 0) {
          cplx *dst = p.env_cur + ((size_t)b * p.nslot_cur + node.env_slot) * ENV_ELEMS;
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 2; ++c) dst[(rq * 4 + r) * CHI + cq + 8 * c] = out[r][c];
        }
        if (node.leaf >= 0) {
          double v = 0.0;
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              const cplx rv = R[(rq * 4 + r) * CHI + cq + 8 * c];
              v += out[r][c].x * rv.x - out[r][c].y * rv.y;
            }
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) p.leafval[(size_t)b * p.nleaf_total + node.leaf] = v;
        }
      }
    }
    __syncwarp();   // S is rewritten by the next parent
  }
  cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// energies[b] = sum_leaf coef[leaf] * value[b, leaf] (fixed-order tree sum),
// per_term[b, t] = value[b, term_leaf[t]]. Failed states give NaN.
// ---------------------------------------------------------------------------
constexpr int REDUCE_THREADS = 256;

__device__ __forceinline__ void reduce_body(const double *__restrict__ lv, const double *__restrict__ coef,
                                            int nleaf, const int32_t *__restrict__ term_leaf, int T, bool ok,
                                            double *__restrict__ energy, double *__restrict__ per_term) {
  __shared__ double part[REDUCE_THREADS];
  const int tid = threadIdx.x;
  double acc = 0.0;
  for (int i = tid; i < nleaf; i += REDUCE_THREADS) acc = fma(coef[i], lv[i], acc);
  part[tid] = acc;
  __syncthreads();
  for (int w = REDUCE_THREADS / 2; w > 0; w >>= 1) {
    if (tid < w) part[tid] += part[tid + w];
    __syncthreads();
  }
  if (tid == 0) *energy = ok ? part[0] : __longlong_as_double(0x7ff8000000000000LL);
  if (per_term != nullptr) {
    for (int t = tid; t < T; t += REDUCE_THREADS)
      per_term[t] = ok ? lv[term_leaf[t]] : __longlong_as_double(0x7ff8000000000000LL);
  }
}

__global__ void __launch_bounds__(REDUCE_THREADS)
reduce_kernel(const double *__restrict__ leafval, const double *__restrict__ coef, int nleaf,
              const int32_t *__restrict__ term_leaf, int T, const int32_t *__restrict__ status,
              double *__restrict__ energies, double *__restrict__ per_term) {
  const int b = blockIdx.x;
  reduce_body(leafval + (size_t)b * nleaf, coef, nleaf, term_leaf, T, status[b] == 0, energies + b,
              per_term ? per_term + (size_t)b * T : nullptr);
}

// Partition sets: partition k = st_part[b] has part_nleaf[k] leaves and
// part_T[k] terms; its leaf coefficients and term -> leaf map sit at
// k * leaf_stride and k * term_stride, the state's leaf values and per-term
// outputs at b * leaf_stride and b * term_stride.
__global__ void __launch_bounds__(REDUCE_THREADS)
reduce_multi_kernel(const double *__restrict__ leafval, const double *__restrict__ coef, int leaf_stride,
                    const int32_t *__restrict__ term_leaf, int term_stride, const int32_t *__restrict__ st_part,
                    const int32_t *__restrict__ part_nleaf, const int32_t *__restrict__ part_T,
                    const int32_t *__restrict__ status, double *__restrict__ energies,
                    double *__restrict__ per_term) {
  const int b = blockIdx.x;
  const int k = st_part[b];
  reduce_body(leafval + (size_t)b * leaf_stride, coef + (size_t)k * leaf_stride, part_nleaf[k],
              term_leaf + (size_t)k * term_stride, part_T[k], status[b] == 0, energies + b,
              per_term ? per_term + (size_t)b * term_stride : nullptr);
}

// Transposed site tensors for the suffix levels of the split evaluation:
// out[b][s][c][i][a] = in[b][s][a][i][c].
__global__ void __launch_bounds__(256)
transpose_sites_kernel(const cplx *__restrict__ in, int n, cplx *__restrict__ out) {
  const size_t base = ((size_t)blockIdx.y * n + blockIdx.x) * SITE_ELEMS;
  for (int e = threadIdx.x; e < SITE_ELEMS; e += 256) {
    const int a = e >> 5, i = (e >> 4) & 1, c = e & 15;
    out[base + c * 32 + i * 16 + a] = in[base + e];
  }
}

// Pair closures of the split evaluation: leafval[b][leaf] = Re sum L o R for
// (prefix slot, suffix slot, leaf) triples; one warp per pair.
constexpr int COMBINE_WARPS = 8;

// A pair closure of the per-term-cut plan: its two operands by region (the level
// region of B x nslot slots starting at slot B x base of its half's buffer) and slot.
struct DevPair {
  int32_t lbase, lnslot, lslot;
  int32_t rbase, rnslot, rslot;
  int32_t leaf, pad;
};
__device__ __forceinline__ size_t pair_offset(int base, int nslot, int slot, int b, int B) {
  return ((size_t)B * base + (size_t)b * nslot + slot) * ENV_ELEMS;
}

// Pair closures of the per-term-cut plan (complex environments).
__global__ void __launch_bounds__(COMBINE_WARPS * 32)
pair_combine_kernel(const cplx *__restrict__ left, const cplx *__restrict__ right, const DevPair *__restrict__ pairs,
                    int npairs, const int32_t *__restrict__ status, double *__restrict__ leafval,
                    int nleaf_total) {
  const int b = blockIdx.y, B = gridDim.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pidx = blockIdx.x * COMBINE_WARPS + warp;
  if (pidx >= npairs) return;
  const DevPair pr = pairs[pidx];
  const cplx *L = left + pair_offset(pr.lbase, pr.lnslot, pr.lslot, b, B);
  const cplx *R = right + pair_offset(pr.rbase, pr.rnslot, pr.rslot, b, B);
  double v = 0.0;
  for (int e = lane; e < ENV_ELEMS; e += 32) {
    const cplx l = L[e], r = R[e];
    v += l.x * r.x - l.y * r.y;
  }
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) leafval[(size_t)b * nleaf_total + pr.leaf] = status[b] == 0 ? v : 0.0;
}
__global__ void __launch_bounds__(COMBINE_WARPS * 32)
split_combine_kernel(const cplx *__restrict__ left, int left_nslot, const cplx *__restrict__ right,
                     int right_nslot, const int32_t *__restrict__ pairs, int npairs,
                     const int32_t *__restrict__ status, double *__restrict__ leafval, int nleaf_total) {
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pidx = blockIdx.x * COMBINE_WARPS + warp;
  if (pidx >= npairs) return;
  const int ls = pairs[3 * pidx], rs = pairs[3 * pidx + 1], leaf = pairs[3 * pidx + 2];
  const cplx *L = left + ((size_t)b * left_nslot + ls) * ENV_ELEMS;
  const cplx *R = right + ((size_t)b * right_nslot + rs) * ENV_ELEMS;
  double v = 0.0;
  for (int e = lane; e < ENV_ELEMS; e += 32) {
    const cplx l = L[e], r = R[e];
    v += l.x * r.x - l.y * r.y;
  }
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) leafval[(size_t)b * nleaf_total + leaf] = status[b] == 0 ? v : 0.0;
}

}  // namespace vqemps
