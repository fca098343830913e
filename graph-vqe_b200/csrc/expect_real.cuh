// Trie levels in real arithmetic, for states whose amplitudes are real.
//
// When every gate of the circuit is real (RY, CX, X, Z, H, SWAP, real U1/U2) and
// the initial state is real, every site tensor A and every identity right
// environment R is real. A trie node's environment is then
//   E = i^k Er,   k = the number of Y codes on the node's path, mod 4 (DevNode.phase),
// with Er real: the transfer E' = sum_ij P_ij A_i^H E A_j (analytic_batch.cuh:4-36
// in the reference, for complex tensors) keeps the factor i^k for I, X and Z and
// multiplies in i for Y. These levels carry Er only:
//   I: A0^T Er A0 + A1^T Er A1        Z: A0^T Er A0 - A1^T Er A1
//   X: A0^T Er A1 + A1^T Er A0        Y: A1^T Er A0 - A0^T Er A1   (phase k + 1)
// and a term's value Re sum_xy E[x][y] R[x][y] is Re(i^k) sum Er o R: zero for
// an odd number of Y's, negated for k = 2. E is Hermitian, so Er is symmetric for
// even k and antisymmetric for odd k; A_x^T Er A_x inherits that, and
// A1^T Er A0 = +-(A0^T Er A1)^T. As in the complex kernels the class products
// form three of four 8 x 8 tiles (the (1,0) tile is +-(0,1)^T) and the X/Y pair
// one product -- but each is ONE real product where the complex kernels issue
// three (Gauss): 56 DMMA issues per one-class parent instead of 168, and the
// environments moved between levels are half the bytes.
//
// Shared tiles hold doubles laid out so that the fragment loads of a half-warp
// (lanes g = 0..3 rows, t = 0..3 columns) fall on 16 distinct 8-byte banks: the
// site panel and S pad their rows to 4 mod 16 doubles; environments keep 16
// doubles per row with the 4-column blocks of row r XOR-swizzled by r mod 4
// (rl_swz), in global memory as well as in shared memory, so the swizzle costs
// no bytes and an environment moves as one contiguous 2,048-byte block.
//
// Tile movement is by the bulk-copy (TMA) engine: real_panels_kernel writes every
// site tensor once per step as a real panel already in the padded shared-memory
// layout, so a CTA stages its site panel and right environment with two 1-D
// cp.async.bulk copies (4,608 + 2,048 bytes), and each warp fetches the next
// parent environment with one 2,048-byte copy; all complete on mbarriers
// (expect_tx), one per CTA and one per warp. Sources are this GPU's memory,
// addresses 16-byte aligned, sizes multiples of 16, and no copy uses cluster
// multicast. Every wait is bounded: a wait that gives up marks the state
// ST_TIMEOUT, waits once more (bounded) for its copies and returns.
#pragma once
#include "common.cuh"
#include "expect.cuh"
#include "expect_mma.cuh"

namespace vqemps {

constexpr int RL_WARPS = 4;
constexpr int RL_A_STRIDE = 36;   // site panel: 16 rows [a] of 32 doubles [i * 16 + c]
constexpr int RL_S_STRIDE = 20;   // S = Er [A_0 | A_1]: [i][a][c], 2 x 16 rows of 16 doubles

constexpr int RL_PANEL = CHI * RL_A_STRIDE;   // doubles per real site panel (4,608 bytes)

// Position of element (r, c) of a real environment (16 x 16, row-major) in the
// swizzled layout: column blocks of four XORed with r mod 4. Two-element runs
// (c even) stay contiguous and 16-byte aligned.
__host__ __device__ __forceinline__ int rl_swz(int r, int c) { return r * CHI + (c ^ ((r & 3) << 2)); }

struct LevelRealSmem {
  double A[RL_PANEL];
  double R[ENV_ELEMS];             // swizzled (rl_swz)
  double E[RL_WARPS][ENV_ELEMS];   // swizzled (rl_swz)
  double S[RL_WARPS][2 * CHI * RL_S_STRIDE];
  uint64_t bar_cta;                 // site panel + right environment
  uint64_t bar_warp[RL_WARPS];      // each warp's parent environment
};

// Re(i^k)
__device__ __forceinline__ double re_ipow(int k) { return (k & 1) ? 0.0 : ((k & 2) ? -1.0 : 1.0); }

// ---- bulk copies completing on an mbarrier ----
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// generic-proxy accesses of shared memory before a bulk copy overwrites it
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Wait until the barrier's phase with the given parity completes; false after
// max_tries attempts (each try_wait may suspend the warp for a while).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int max_tries) {
  for (int i = 0; i < max_tries; ++i) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
constexpr int RL_WAIT_TRIES = 1 << 20;

// The parent environment of group grp into E, completing the warp's barrier
// phase: a real environment of the previous level or, for a suffix root, the
// real identity right environment R_{s+1} (one 2,048-byte bulk copy issued by
// lane 0; both are stored swizzled), or the 1 x 1 vacuum (plain stores, then a
// plain arrive; element (0, 0) sits at position 0 in either layout).
// The caller has finished reading E (and synchronised the warp).
__device__ __forceinline__ void stage_parent_real(const LevelParams &p, int b, const DevGroup &grp, double *E,
                                                  uint64_t *bar, int lane) {
  if (grp.parent_slot < 0 && !p.suffix) {
    for (int e = lane; e < ENV_ELEMS; e += 32) E[e] = e == 0 ? 1.0 : 0.0;
    __syncwarp();
    if (lane == 0) mbar_arrive(bar);
    return;
  }
  const double *src = grp.parent_slot < 0
                          ? p.right_real + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS
                          : reinterpret_cast<const double *>(p.env_prev) +
                                ((size_t)b * p.nslot_prev + grp.parent_slot) * ENV_ELEMS;
  if (lane == 0) {
    async_proxy_fence();
    mbar_arrive_expect_tx(bar, ENV_ELEMS * sizeof(double));
    bulk_copy_g2s(E, src, ENV_ELEMS * sizeof(double), bar);
  }
}

// The X/Y class product t0 = A_0^T S_1 over all four 8 x 8 output tiles.
__device__ __forceinline__ void class_tiles_real_xy(const double *A, const double *S, double (&acc)[2][2][2],
                                                    int g, int t) {
#pragma unroll
  for (int rt = 0; rt < 2; ++rt)
#pragma unroll
    for (int ct = 0; ct < 2; ++ct) acc[rt][ct][0] = acc[rt][ct][1] = 0.0;
#pragma unroll
  for (int ks = 0; ks < 4; ++ks) {
    double x[2], yv[2];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt) x[rt] = A[(ks * 4 + t) * RL_A_STRIDE + rt * 8 + g];
#pragma unroll
    for (int ct = 0; ct < 2; ++ct) yv[ct] = S[(CHI + ks * 4 + t) * RL_S_STRIDE + ct * 8 + g];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 2; ++ct) dmma(acc[rt][ct][0], acc[rt][ct][1], x[rt], yv[ct]);
  }
}

// The I/Z class pair in one pass: a = A_0^T S_0 and c = A_1^T S_1 over the
// tiles (0,0), (0,1), (1,1) -- six independent accumulators per k-step, so
// consecutive DMMA issues of a warp do not wait on each other.
__device__ __forceinline__ void class_tiles_real_iz(const double *A, const double *S, double (&a)[2][2][2],
                                                    double (&c)[2][2][2], int g, int t) {
#pragma unroll
  for (int rt = 0; rt < 2; ++rt)
#pragma unroll
    for (int ct = 0; ct < 2; ++ct) a[rt][ct][0] = a[rt][ct][1] = c[rt][ct][0] = c[rt][ct][1] = 0.0;
#pragma unroll
  for (int ks = 0; ks < 4; ++ks) {
    double x0[2], x1[2], y0[2], y1[2];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt) {
      x0[rt] = A[(ks * 4 + t) * RL_A_STRIDE + rt * 8 + g];
      x1[rt] = A[(ks * 4 + t) * RL_A_STRIDE + CHI + rt * 8 + g];
    }
#pragma unroll
    for (int ct = 0; ct < 2; ++ct) {
      y0[ct] = S[(ks * 4 + t) * RL_S_STRIDE + ct * 8 + g];
      y1[ct] = S[(CHI + ks * 4 + t) * RL_S_STRIDE + ct * 8 + g];
    }
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = rt; ct < 2; ++ct) {
        dmma(a[rt][ct][0], a[rt][ct][1], x0[rt], y0[ct]);
        dmma(c[rt][ct][0], c[rt][ct][1], x1[rt], y1[ct]);
      }
  }
}

// One trie level for B states (uniform batch: state blockIdx.y, groups
// interleaved over the grid, groups_per_warp each), environments as real parts.
// Five CTAs per SM (96 registers, 35 KB of shared memory each): measured 3 %
// faster at 40 qubits / B = 256 than four (120 registers).
__global__ void __launch_bounds__(RL_WARPS * 32, 5)
level_real_pf_kernel(LevelParams p, int groups_per_warp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LevelRealSmem &sm = *reinterpret_cast<LevelRealSmem *>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int b = p.flip ? (int)(gridDim.y - 1 - blockIdx.y) : (int)blockIdx.y;
  const int stride = gridDim.x * RL_WARPS;
  const int first = blockIdx.x * RL_WARPS + warp;
  int count = 0;
  if (first < p.ngroups) count = min(groups_per_warp, (p.ngroups - first + stride - 1) / stride);
  if (threadIdx.x == 0) {
    mbar_init(&sm.bar_cta, 1);
    for (int w = 0; w < RL_WARPS; ++w) mbar_init(&sm.bar_warp[w], 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(&sm.bar_cta, (RL_PANEL + ENV_ELEMS) * sizeof(double));
    bulk_copy_g2s(sm.A, p.panels + ((size_t)b * p.n + p.s) * RL_PANEL, RL_PANEL * sizeof(double), &sm.bar_cta);
    bulk_copy_g2s(sm.R, p.right_real + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS, ENV_ELEMS * sizeof(double),
                  &sm.bar_cta);
  }
  if (!mbar_wait(&sm.bar_cta, 0, RL_WAIT_TRIES)) {
    if (threadIdx.x == 0) p.status[b] = ST_TIMEOUT;
    mbar_wait(&sm.bar_cta, 0, RL_WAIT_TRIES);
    return;
  }
  const double *A = sm.A;
  const double *R = sm.R;
  double *E = sm.E[warp];
  double *S = sm.S[warp];
  uint64_t *bar = &sm.bar_warp[warp];
  unsigned parity = 0;
  double *env_cur = reinterpret_cast<double *>(p.env_cur);
  const int g = lane >> 2, t = lane & 3;
  if (count == 0) return;
  // Group and node records are software pipelined: the next group's record is
  // loaded while this group's first half runs (its parent slot addresses the
  // next prefetch), and its children's node records -- at most four, one per
  // lane, read back with shuffles -- at the end of this group. No global load
  // of plan metadata then sits on the warp's critical path.
  DevGroup grp = p.groups[first];
  DevNode nd{};
  if (lane < grp.nchild) nd = p.nodes[grp.child_begin + lane];
  stage_parent_real(p, b, grp, E, bar, lane);
  for (int k = 0; k < count; ++k) {
    const int gidx = first + k * stride;
    const bool more = k + 1 < count;
    DevGroup grp_next = grp;
    if (more) grp_next = p.groups[gidx + stride];
    if (!mbar_wait(bar, parity, RL_WAIT_TRIES)) {
      if (lane == 0) p.status[b] = ST_TIMEOUT;
      mbar_wait(bar, parity, RL_WAIT_TRIES);
      return;
    }
    parity ^= 1u;
    // ---- S = Er [A_0 | A_1] (16 x 32): 32 DMMA issues
    {
      double sacc[2][4][2];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) sacc[rt][ct][0] = sacc[rt][ct][1] = 0.0;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        double ef[2], pf[4];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt) ef[rt] = E[rl_swz(rt * 8 + g, ks * 4 + t)];
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) pf[ct] = A[(ks * 4 + t) * RL_A_STRIDE + ct * 8 + g];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 4; ++ct) dmma(sacc[rt][ct][0], sacc[rt][ct][1], ef[rt], pf[ct]);
      }
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 4; ++ct)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int col = ct * 8 + 2 * t + j;
            S[((col >> 4) * CHI + rt * 8 + g) * RL_S_STRIDE + (col & 15)] = sacc[rt][ct][j];
          }
    }
    __syncwarp();   // Er is dead and S is complete: fetch the next parent
    if (more) stage_parent_real(p, b, grp_next, E, bar, lane);
    // the parent's phase (from its first child): symmetric Er for even, antisymmetric for odd
    const int c0 = __shfl_sync(0xffffffffu, nd.code, 0), k0 = __shfl_sync(0xffffffffu, nd.phase, 0);
    const int kp = (k0 - (c0 == 2 ? 1 : 0)) & 3;
    const double sp = (kp & 1) ? -1.0 : 1.0;
    for (int cls = 0; cls < 2; ++cls) {
      if (!(grp.classes & (1 << cls))) continue;
      // I/Z: t0 = A_0^T S_0, t1 = A_1^T S_1 (tiles (0,0), (0,1), (1,1));
      // X/Y: t0 = A_0^T S_1 (four tiles), t1 = A_1^T S_0 = sp t0^T through the panel
      double a[2][2][2], c[2][2][2];
      if (cls == 0) {
        class_tiles_real_iz(A, S, a, c, g, t);
      } else {
        class_tiles_real_xy(A, S, a, g, t);
        __syncwarp();   // the panel is consumed: t0 goes into its place
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) S[(rt * 8 + g) * RL_S_STRIDE + ct * 8 + 2 * t + j] = a[rt][ct][j];
        __syncwarp();
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = rt; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) c[rt][ct][j] = sp * S[(ct * 8 + 2 * t + j) * RL_S_STRIDE + rt * 8 + g];
      }
      for (int ci = 0; ci < grp.nchild; ++ci) {
        DevNode node;
        node.code = __shfl_sync(0xffffffffu, nd.code, ci);
        node.env_slot = __shfl_sync(0xffffffffu, nd.env_slot, ci);
        node.leaf = __shfl_sync(0xffffffffu, nd.leaf, ci);
        node.phase = __shfl_sync(0xffffffffu, nd.phase, ci);
        const bool iz = (node.code == 0 || node.code == 3);
        if (iz != (cls == 0)) continue;
        // child symmetry: the (1,0) tile is sc times the transposed (0,1) tile
        const double sc = (node.phase & 1) ? -1.0 : 1.0;
        double out[2][2][2];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = rt; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              const double t0 = a[rt][ct][j], t1 = c[rt][ct][j];
              out[rt][ct][j] = (node.code == 0 || node.code == 1) ? t0 + t1 : (node.code == 3 ? t0 - t1 : t1 - t0);
            }
        if (node.env_slot >= 0) {
          double *dst = env_cur + ((size_t)b * p.nslot_cur + node.env_slot) * ENV_ELEMS;
#pragma unroll
          for (int rt = 0; rt < 2; ++rt)
#pragma unroll
            for (int ct = rt; ct < 2; ++ct)
              *reinterpret_cast<double2 *>(dst + rl_swz(rt * 8 + g, ct * 8 + 2 * t)) =
                  make_double2(out[rt][ct][0], out[rt][ct][1]);
#pragma unroll
          for (int j = 0; j < 2; ++j) dst[rl_swz(8 + 2 * t + j, g)] = sc * out[0][1][j];
        }
        if (node.leaf >= 0) {
          const double w = re_ipow(node.phase);
          double v = 0.0;
          if (w != 0.0) {
#pragma unroll
            for (int rt = 0; rt < 2; ++rt)
#pragma unroll
              for (int ct = rt; ct < 2; ++ct)
#pragma unroll
                for (int j = 0; j < 2; ++j) v += out[rt][ct][j] * R[rl_swz(rt * 8 + g, ct * 8 + 2 * t + j)];
#pragma unroll
            for (int j = 0; j < 2; ++j) v += sc * out[0][1][j] * R[rl_swz(8 + 2 * t + j, g)];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          }
          if (lane == 0) p.leafval[(size_t)b * p.nleaf_total + node.leaf] = w * v;
        }
      }
    }
    __syncwarp();   // S is rewritten by the next parent
    grp = grp_next;
    if (more && lane < grp.nchild) nd = p.nodes[grp.child_begin + lane];
  }
}

// The pair closures of the split evaluation on real-part environments:
// value = Re(i^(prefix phase + suffix phase)) sum_xy L[x][y] R[x][y] (pair_sign).
// A pair with a nonzero sign has an even phase sum, so L and R are both
// symmetric or both antisymmetric and L[y][x] R[y][x] = L[x][y] R[x][y]: the sum
// is the diagonal plus twice the upper triangle. A warp reads only the 4-column
// blocks that reach the diagonal or above -- 40 of the 64 blocks of 32 bytes
// (both sides are stored swizzled alike, rl_swz) -- 5/8 of the bytes.
__device__ __forceinline__ double real_pair_dot(const double *L, const double *R, int lane) {
  double v = 0.0;
  // block q of the upper part: rows 0-3 four blocks each, rows 4-7 three (from
  // block 1), rows 8-11 two (from 2), rows 12-15 one (block 3)
  for (int q = lane; q < 40; q += 32) {
    int r, lb;
    if (q < 16) { r = q >> 2; lb = q & 3; }
    else if (q < 28) { r = 4 + (q - 16) / 3; lb = 1 + (q - 16) % 3; }
    else if (q < 36) { r = 8 + ((q - 28) >> 1); lb = 2 + ((q - 28) & 1); }
    else { r = 12 + (q - 36); lb = 3; }
    const int off = rl_swz(r, 4 * lb);
    const double2 l0 = *reinterpret_cast<const double2 *>(L + off);
    const double2 l1 = *reinterpret_cast<const double2 *>(L + off + 2);
    const double2 r0 = *reinterpret_cast<const double2 *>(R + off);
    const double2 r1 = *reinterpret_cast<const double2 *>(R + off + 2);
    const double lv[4] = {l0.x, l0.y, l1.x, l1.y}, rv[4] = {r0.x, r0.y, r1.x, r1.y};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = 4 * lb + j;
      const double wt = c > r ? 2.0 : (c == r ? 1.0 : 0.0);
      v = fma(wt * lv[j], rv[j], v);
    }
  }
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(COMBINE_WARPS * 32)
split_combine_real_kernel(const double *__restrict__ left, int left_nslot, const double *__restrict__ right,
                          int right_nslot, const int32_t *__restrict__ pairs, const double *__restrict__ pair_sign,
                          int npairs, const int32_t *__restrict__ status, double *__restrict__ leafval,
                          int nleaf_total) {
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pidx = blockIdx.x * COMBINE_WARPS + warp;
  if (pidx >= npairs) return;
  const int ls = pairs[3 * pidx], rs = pairs[3 * pidx + 1], leaf = pairs[3 * pidx + 2];
  const double w = pair_sign[pidx];
  double v = 0.0;
  if (w != 0.0)
    v = real_pair_dot(left + ((size_t)b * left_nslot + ls) * ENV_ELEMS,
                      right + ((size_t)b * right_nslot + rs) * ENV_ELEMS, lane);
  if (lane == 0) leafval[(size_t)b * nleaf_total + leaf] = status[b] == 0 ? w * v : 0.0;
}

// The same closures for the per-term-cut plan (operands by level region).
__global__ void __launch_bounds__(COMBINE_WARPS * 32)
pair_combine_real_kernel(const double *__restrict__ left, const double *__restrict__ right,
                         const DevPair *__restrict__ pairs, const double *__restrict__ pair_sign, int npairs,
                         const int32_t *__restrict__ status, double *__restrict__ leafval, int nleaf_total) {
  const int b = blockIdx.y, B = gridDim.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pidx = blockIdx.x * COMBINE_WARPS + warp;
  if (pidx >= npairs) return;
  const DevPair pr = pairs[pidx];
  const double w = pair_sign[pidx];
  double v = 0.0;
  if (w != 0.0)
    v = real_pair_dot(left + pair_offset(pr.lbase, pr.lnslot, pr.lslot, b, B),
                      right + pair_offset(pr.rbase, pr.rnslot, pr.rslot, b, B), lane);
  if (lane == 0) leafval[(size_t)b * nleaf_total + pr.leaf] = status[b] == 0 ? w * v : 0.0;
}

// Real site panels of one step: panel (b, s) holds the real parts of site s of
// state b in the padded shared-memory layout of level_real_pf_kernel (row a,
// column i * CHI + c, stride RL_A_STRIDE; padding columns zero). transposed:
// the panel of A^T[c][i][a] = A[a][i][c] (the suffix levels).
__global__ void __launch_bounds__(256)
real_panels_kernel(const cplx *__restrict__ sites, int n, int transposed, double *__restrict__ panels) {
  const size_t base = (size_t)blockIdx.y * n + blockIdx.x;
  const cplx *a = sites + base * SITE_ELEMS;
  double *out = panels + base * RL_PANEL;
  for (int e = threadIdx.x; e < RL_PANEL; e += 256) {
    const int row = e / RL_A_STRIDE, col = e - row * RL_A_STRIDE;
    double v = 0.0;
    if (col < 2 * CHI) {
      const int i = col >> 4, c = col & 15;
      v = transposed ? a[c * 2 * CHI + i * CHI + row].x : a[row * 2 * CHI + i * CHI + c].x;
    }
    out[e] = v;
  }
}

// Identity right environments of states with real amplitudes (right_env_kernel
// in real arithmetic): R_n = 1, R_s[b][b'] = sum_{i,c,c'} A[b][i][c] R_{s+1}[c][c']
// A[b'][i][c'] with A real, one CTA per state. The outputs are those of
// right_env_kernel -- R and the branch matrices M_i as complex numbers with zero
// imaginary parts, the norm in the identity leaf -- plus the real parts of every
// R_s in right_real (swizzled, rl_swz), the copy the real-arithmetic levels
// stage, and -- when panels / panels_t are non-null -- every site's real panel
// and transposed panel (real_panels_kernel's output) from the staged tile, so
// the levels need no separate panel pass. The site tile is
// padded to 33 doubles per row, so the first contraction's 16 rows of a
// half-warp fall on distinct banks.
__global__ void __launch_bounds__(RIGHT_THREADS)
right_env_real_kernel(const cplx *__restrict__ sites, int n, cplx *__restrict__ right,
                      cplx *__restrict__ branch, const int32_t *__restrict__ status,
                      double *__restrict__ leafval, int nleaf_total, int identity_leaf,
                      double *__restrict__ right_real, double *__restrict__ panels,
                      double *__restrict__ panels_t) {
  constexpr int AS = 2 * CHI + 1;
  __shared__ double A[CHI * AS];
  __shared__ double R[ENV_ELEMS];
  __shared__ double T[2 * ENV_ELEMS];
  const int b = blockIdx.x, tid = threadIdx.x;
  const cplx *sb = sites + (size_t)b * n * SITE_ELEMS;
  cplx *rb = right + (size_t)b * (n + 1) * ENV_ELEMS;
  double *rr = right_real + (size_t)b * (n + 1) * ENV_ELEMS;
  cplx *mbase = branch ? branch + (size_t)b * n * 2 * ENV_ELEMS : nullptr;
  R[tid] = tid == 0 ? 1.0 : 0.0;
  rb[(size_t)n * ENV_ELEMS + tid] = cmake(R[tid], 0.0);
  rr[(size_t)n * ENV_ELEMS + rl_swz(tid >> 4, tid & 15)] = R[tid];
  for (int s = n - 1; s >= 0; --s) {
    for (int e = tid; e < SITE_ELEMS; e += RIGHT_THREADS) A[(e >> 5) * AS + (e & 31)] = sb[(size_t)s * SITE_ELEMS + e].x;
    __syncthreads();
    if (panels != nullptr) {
      // panel row a, column i * CHI + c: A[a][i][c]; transposed: row c, column i * CHI + a
      double *pn = panels + ((size_t)b * n + s) * RL_PANEL;
      double *pt = panels_t != nullptr ? panels_t + ((size_t)b * n + s) * RL_PANEL : nullptr;
      for (int e = tid; e < RL_PANEL; e += RIGHT_THREADS) {
        const int row = e / RL_A_STRIDE, col = e - row * RL_A_STRIDE;
        const bool in = col < 2 * CHI;
        pn[e] = in ? A[row * AS + col] : 0.0;
        if (pt != nullptr) pt[e] = in ? A[(col & 15) * AS + (col >> 4) * CHI + row] : 0.0;
      }
    }
    // T_i[c][b'] = sum_c' R[c][c'] A[b'][i][c']
    {
      const int c = tid >> 4, bp = tid & 15;
      double t0 = 0.0, t1 = 0.0;
      for (int cp = 0; cp < CHI; ++cp) {
        const double r = R[c * CHI + cp];
        t0 = fma(r, A[bp * AS + cp], t0);
        t1 = fma(r, A[bp * AS + CHI + cp], t1);
      }
      T[c * CHI + bp] = t0;
      T[ENV_ELEMS + c * CHI + bp] = t1;
    }
    __syncthreads();
    // R_s[bb][b'] = sum_i M_i[bb][b'],  M_i[bb][b'] = sum_c A[bb][i][c] T_i[c][b']
    {
      const int bb = tid >> 4, bp = tid & 15;
      double m0 = 0.0, m1 = 0.0;
      for (int c = 0; c < CHI; ++c) {
        m0 = fma(A[bb * AS + c], T[c * CHI + bp], m0);
        m1 = fma(A[bb * AS + CHI + c], T[ENV_ELEMS + c * CHI + bp], m1);
      }
      const double acc = m0 + m1;
      R[tid] = acc;
      rb[(size_t)s * ENV_ELEMS + tid] = cmake(acc, 0.0);
      rr[(size_t)s * ENV_ELEMS + rl_swz(bb, bp)] = acc;
      if (mbase != nullptr) {
        cplx *mb = mbase + (size_t)s * 2 * ENV_ELEMS;
        mb[tid] = cmake(m0, 0.0);
        mb[ENV_ELEMS + tid] = cmake(m1, 0.0);
      }
    }
    __syncthreads();
  }
  if (identity_leaf >= 0 && leafval != nullptr && tid == 0)
    leafval[(size_t)b * nleaf_total + identity_leaf] = status[b] == 0 ? R[0] : 0.0;
}

// Real parts of count / ENV_ELEMS complex environments, each stored swizzled (rl_swz).
__global__ void __launch_bounds__(256)
real_parts_kernel(const cplx *__restrict__ in, size_t count, double *__restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * 256 + threadIdx.x; i < count; i += (size_t)gridDim.x * 256) {
    const int e = (int)(i % ENV_ELEMS);
    out[i - e + rl_swz(e >> 4, e & 15)] = in[i].x;
  }
}

}  // namespace vqemps
