// Gradient trie levels on the FP64 tensor cores (DMMA, mma.sync m8n8k4 .f64).
//
// Same work, outputs and CTA partition as grad_fwd_level_kernel /
// grad_bwd_level_kernel (gradient.cuh): CTA x of state b owns groups
// 16x .. 16x + 15 of the level, warp w takes groups w, w + 4, ...; per-CTA
// partial sums (leaf sums forward, site cotangents backward) are combined by
// partial_sum_kernel in a fixed order. Complex products are four real DMMA
// products over 8 x 8 output tiles (expect_mma.cuh gives the fragment layout
// and the padded shared-memory strides).
#pragma once
#include "common.cuh"
#include "expect.cuh"
#include "expect_mma.cuh"
#include "gradient.cuh"

namespace vqemps {

struct GradFwdMmaSmem {
  cplx A[CHI * MMA_A_STRIDE];
  cplx R[ENV_ELEMS];
  cplx E[GLEVEL_WARPS][CHI * MMA_E_STRIDE];
  cplx S[GLEVEL_WARPS][2 * CHI * MMA_S_STRIDE];
  cplx L[GLEVEL_WARPS][ENV_ELEMS];
};

__device__ __forceinline__ void grad_stage_parent(const GradLevelParams &p, int b, int g, cplx *E, int lane) {
  const DevGroup grp = p.groups[g];
  if (grp.parent_slot < 0 && p.suffix) {
    const cplx *src = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
    for (int e = lane; e < ENV_ELEMS; e += 32) cp_async16(E + (e >> 4) * MMA_E_STRIDE + (e & 15), src + e);
  } else if (grp.parent_slot < 0) {
    for (int e = lane; e < ENV_ELEMS; e += 32)
      E[(e >> 4) * MMA_E_STRIDE + (e & 15)] = cmake(e == 0 ? 1.0 : 0.0, 0.0);
  } else {
    const cplx *src = p.env_prev + (size_t)b * p.prev_stride + (size_t)grp.parent_slot * ENV_ELEMS;
    for (int e = lane; e < ENV_ELEMS; e += 32) cp_async16(E + (e >> 4) * MMA_E_STRIDE + (e & 15), src + e);
  }
}

// S panel [S_0 | S_1] = E [A_0 | A_1] (16 x 32, K = 16) into padded S[i][row][col];
// KIND 1 (Gauss): three real products per complex product (k1 = Yr (Xr + Xi),
// k2 = Xr (Yi - Yr), k3 = Xi (Yr + Yi); Re = k1 - k3, Im = k1 + k2); KIND 0:
// four.
template <int KIND = 0>
__device__ __forceinline__ void mma_panel_EA(const cplx *E, const cplx *A, cplx *S, int g, int t) {
  constexpr bool GAUSS = KIND == 1;
  double sr[2][4][2], si[2][4][2], s3[GAUSS ? 2 : 1][4][2];
#pragma unroll
  for (int rt = 0; rt < 2; ++rt)
#pragma unroll
    for (int ct = 0; ct < 4; ++ct) { sr[rt][ct][0] = sr[rt][ct][1] = 0.0; si[rt][ct][0] = si[rt][ct][1] = 0.0; }
  if constexpr (GAUSS) {
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) s3[rt][ct][0] = s3[rt][ct][1] = 0.0;
  }
#pragma unroll
  for (int ks = 0; ks < 4; ++ks) {
    cplx ef[2], pf[4];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt) ef[rt] = E[(rt * 8 + g) * MMA_E_STRIDE + ks * 4 + t];
#pragma unroll
    for (int ct = 0; ct < 4; ++ct) pf[ct] = A[(ks * 4 + t) * MMA_A_STRIDE + ct * 8 + g];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt) {
      const double er = ef[rt].x, ei = ef[rt].y, nei = -ef[rt].y;
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) {
        if constexpr (GAUSS) {
          dmma(sr[rt][ct][0], sr[rt][ct][1], er + ei, pf[ct].x);                 // k1
          dmma(si[rt][ct][0], si[rt][ct][1], er, pf[ct].y - pf[ct].x);           // k2
          dmma(s3[rt][ct][0], s3[rt][ct][1], ei, pf[ct].x + pf[ct].y);           // k3
        } else {
          dmma(sr[rt][ct][0], sr[rt][ct][1], er, pf[ct].x);
          dmma(sr[rt][ct][0], sr[rt][ct][1], nei, pf[ct].y);
          dmma(si[rt][ct][0], si[rt][ct][1], er, pf[ct].y);
          dmma(si[rt][ct][0], si[rt][ct][1], ei, pf[ct].x);
        }
      }
    }
  }
#pragma unroll
  for (int rt = 0; rt < 2; ++rt)
#pragma unroll
    for (int ct = 0; ct < 4; ++ct)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int col = ct * 8 + 2 * t + j;
        cplx v;
        if constexpr (GAUSS) v = cmake(sr[rt][ct][j] - s3[rt][ct][j], sr[rt][ct][j] + si[rt][ct][j]);
        else v = cmake(sr[rt][ct][j], si[rt][ct][j]);
        S[((col >> 4) * CHI + rt * 8 + g) * MMA_S_STRIDE + (col & 15)] = v;
      }
}

template <int KIND>
__device__ __forceinline__ void grad_fwd_level_mma_body(const GradLevelParams &p, unsigned char *smem_raw) {
  GradFwdMmaSmem &sm = *reinterpret_cast<GradFwdMmaSmem *>(smem_raw);
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {
    const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
    const cplx *rg = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
    for (int e = threadIdx.x; e < SITE_ELEMS; e += GLEVEL_WARPS * 32) sm.A[(e >> 5) * MMA_A_STRIDE + (e & 31)] = ag[e];
    for (int e = threadIdx.x; e < ENV_ELEMS; e += GLEVEL_WARPS * 32) sm.R[e] = rg[e];
    for (int e = lane; e < ENV_ELEMS; e += 32) sm.L[warp][e] = cmake(0, 0);
  }
  __syncthreads();
  const cplx *A = sm.A;
  const cplx *R = sm.R;
  cplx *E = sm.E[warp];
  cplx *S = sm.S[warp];
  cplx *L = sm.L[warp];
  const int g = lane >> 2, t = lane & 3;
  const int per_cta = GLEVEL_WARPS * GROUPS_PER_WARP;
  const int g0 = blockIdx.x * per_cta;
  const int g1 = min(g0 + per_cta, p.ngroups);
  int gidx = g0 + warp;
  if (gidx < g1) {
    grad_stage_parent(p, b, gidx, E, lane);
    cp_async_commit();
  }
  for (; gidx < g1; gidx += GLEVEL_WARPS) {
    cp_async_wait<0>();
    __syncwarp();
    const DevGroup grp = p.groups[gidx];
    mma_panel_EA<KIND>(E, A, S, g, t);
    __syncwarp();   // E is dead and S complete: prefetch the next parent
    if (gidx + GLEVEL_WARPS < g1) grad_stage_parent(p, b, gidx + GLEVEL_WARPS, E, lane);
    cp_async_commit();
    for (int cls = 0; cls < 2; ++cls) {
      if (!(grp.classes & (1 << cls))) continue;
      // Hermitian children: tiles (0,0), (0,1), (1,1) formed, (1,0) = (0,1)^H;
      // X/Y: t1 = A_1^H S_0 = t0^H through the S panel (as level_mma_pf_body).
      double ar[2][2][2], ai[2][2][2], br[2][2][2], bi[2][2][2];
      if (cls == 0) {
        class_tiles<KIND, true>(A, 0, S, 0, ar, ai, g, t);
        class_tiles<KIND, true>(A, CHI, S, 1, br, bi, g, t);
      } else {
        class_tiles<KIND, false>(A, 0, S, 1, ar, ai, g, t);
        __syncwarp();
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j)
              S[(rt * 8 + g) * MMA_S_STRIDE + ct * 8 + 2 * t + j] = cmake(ar[rt][ct][j], ai[rt][ct][j]);
        __syncwarp();
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = rt; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              const cplx v = S[(ct * 8 + 2 * t + j) * MMA_S_STRIDE + rt * 8 + g];
              br[rt][ct][j] = v.x;
              bi[rt][ct][j] = -v.y;
            }
      }
      for (int ci = 0; ci < grp.nchild; ++ci) {
        const DevNode node = p.nodes[grp.child_begin + ci];
        const bool iz = (node.code == 0 || node.code == 3);
        if (iz != (cls == 0)) continue;
        cplx out[2][2][2];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = rt; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              const cplx t0 = cmake(ar[rt][ct][j], ai[rt][ct][j]);
              const cplx t1 = cmake(br[rt][ct][j], bi[rt][ct][j]);
              if (node.code == 0 || node.code == 1) out[rt][ct][j] = cadd(t0, t1);
              else if (node.code == 3) out[rt][ct][j] = csub(t0, t1);
              else { const cplx d = csub(t1, t0); out[rt][ct][j] = cmake(-d.y, d.x); }
            }
        // out[1][0][j]: the (1,0)-tile element this lane owns, [8 + 2t + j][g]
        out[1][0][0] = cconj(out[0][1][0]);
        out[1][0][1] = cconj(out[0][1][1]);
        if (node.env_slot >= 0) {
          cplx *dst = p.env_cur + (size_t)b * p.cur_stride + (size_t)node.env_slot * ENV_ELEMS;
#pragma unroll
          for (int rt = 0; rt < 2; ++rt)
#pragma unroll
            for (int ct = rt; ct < 2; ++ct)
#pragma unroll
              for (int j = 0; j < 2; ++j) dst[(rt * 8 + g) * CHI + ct * 8 + 2 * t + j] = out[rt][ct][j];
#pragma unroll
          for (int j = 0; j < 2; ++j) dst[(8 + 2 * t + j) * CHI + g] = out[1][0][j];
        }
        if (node.leaf >= 0 && p.leaf_work) {
          const double cf = p.leaf_coef[node.leaf];
          double v = 0.0;
#pragma unroll
          for (int rt = 0; rt < 2; ++rt)
#pragma unroll
            for (int ct = rt; ct < 2; ++ct)
#pragma unroll
              for (int j = 0; j < 2; ++j) {
                const int idx = (rt * 8 + g) * CHI + ct * 8 + 2 * t + j;
                const cplx rv = R[idx];
                v += out[rt][ct][j].x * rv.x - out[rt][ct][j].y * rv.y;
                L[idx] = cadd(L[idx], cscale(out[rt][ct][j], cf));
              }
#pragma unroll
          for (int j = 0; j < 2; ++j) {   // the (1,0) tile
            const int idx = (8 + 2 * t + j) * CHI + g;
            const cplx rv = R[idx];
            v += out[1][0][j].x * rv.x - out[1][0][j].y * rv.y;
            L[idx] = cadd(L[idx], cscale(out[1][0][j], cf));
          }
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) p.leafval[(size_t)b * p.nleaf + node.leaf] = v;
        }
      }
    }
    __syncwarp();   // S is rewritten by the next parent
  }
  cp_async_wait<0>();
  __syncthreads();
  if (!p.leaf_work) return;
  cplx *dst = p.partial + ((size_t)b * gridDim.x + blockIdx.x) * ENV_ELEMS;
  for (int e = threadIdx.x; e < ENV_ELEMS; e += GLEVEL_WARPS * 32) {
    cplx acc = sm.L[0][e];
    for (int w = 1; w < GLEVEL_WARPS; ++w) acc = cadd(acc, sm.L[w][e]);
    dst[e] = acc;
  }
}

__global__ void __launch_bounds__(GLEVEL_WARPS * 32, 2)
grad_fwd_level_mma_kernel(GradLevelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  grad_fwd_level_mma_body<0>(p, smem_raw);
}

// Forward gradient level with Gauss's three-product complex multiply.
__global__ void __launch_bounds__(GLEVEL_WARPS * 32, 2)
grad_fwd_level_mma3_kernel(GradLevelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  grad_fwd_level_mma_body<1>(p, smem_raw);
}



// ---------------------------------------------------------------------------
// backward level on DMMA. Per group (parent E, site A = [A_0 A_1]):
//   S_i = E A_i;  per Pauli class, D pair from the children's cotangents and
//   leaf weights (cls 0: D_0 = xa + xb, D_1 = xa - xb with xa, xb of I / Z;
//   cls 1: D_0 = xa + i xb, D_1 = xa - i xb with xa, xb of X / Y);
//   Abar_o += 2 S_{src(o)} D_{src(o)},  Y_o += A_{src(o)} D_{src(o)},
//   src(o) = o (cls 0) or 1 - o (cls 1);  Ebar_parent = sum_i Y_i A_i^H.
// The site cotangent accumulates in registers over the warp's groups; the
// warps' panels are combined in a fixed order at the end.
// ---------------------------------------------------------------------------
struct GradBwdMmaSmem {
  cplx A[CHI * MMA_A_STRIDE];
  cplx R[ENV_ELEMS];
  cplx E[GLEVEL_WARPS][CHI * MMA_E_STRIDE];
  cplx S[GLEVEL_WARPS][2 * CHI * MMA_S_STRIDE];   // S panel, later the Y panel
  cplx D[GLEVEL_WARPS][2 * CHI * MMA_S_STRIDE];   // the class's D pair [d][k][c]
};

__device__ __forceinline__ void grad_bwd_level_mma_body(const GradLevelParams &p, unsigned char *smem_raw) {
  GradBwdMmaSmem &sm = *reinterpret_cast<GradBwdMmaSmem *>(smem_raw);
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {
    const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
    const cplx *rg = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
    for (int e = threadIdx.x; e < SITE_ELEMS; e += GLEVEL_WARPS * 32) sm.A[(e >> 5) * MMA_A_STRIDE + (e & 31)] = ag[e];
    for (int e = threadIdx.x; e < ENV_ELEMS; e += GLEVEL_WARPS * 32) sm.R[e] = rg[e];
  }
  __syncthreads();
  const cplx *A = sm.A;
  const cplx *R = sm.R;
  cplx *E = sm.E[warp];
  cplx *S = sm.S[warp];
  cplx *D = sm.D[warp];
  const int g = lane >> 2, t = lane & 3;
  // site cotangent panel of this warp: rows rt * 8 + g, cols ct * 8 + 2t + j of [Abar_0 | Abar_1]
  double abr[2][4][2], abi[2][4][2];
#pragma unroll
  for (int rt = 0; rt < 2; ++rt)
#pragma unroll
    for (int ct = 0; ct < 4; ++ct) { abr[rt][ct][0] = abr[rt][ct][1] = 0.0; abi[rt][ct][0] = abi[rt][ct][1] = 0.0; }
  const int per_cta = GLEVEL_WARPS * GROUPS_PER_WARP;
  const int g0 = blockIdx.x * per_cta;
  const int g1 = min(g0 + per_cta, p.ngroups);
  int gidx = g0 + warp;
  if (gidx < g1) {
    grad_stage_parent(p, b, gidx, E, lane);
    cp_async_commit();
  }
  for (; gidx < g1; gidx += GLEVEL_WARPS) {
    cp_async_wait<0>();
    __syncwarp();
    const DevGroup grp = p.groups[gidx];
    int idx_child[4] = {-1, -1, -1, -1};
    for (int ci = 0; ci < grp.nchild; ++ci) idx_child[p.nodes[grp.child_begin + ci].code] = grp.child_begin + ci;
    // Y_o = sum over classes of A_src(o) D_src(o)
    double yr[2][4][2], yi[2][4][2];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) { yr[rt][ct][0] = yr[rt][ct][1] = 0.0; yi[rt][ct][0] = yi[rt][ct][1] = 0.0; }
    for (int cls = 0; cls < 2; ++cls) {
      if (!(grp.classes & (1 << cls))) continue;
      const int ca = idx_child[cls == 0 ? 0 : 1], cbx = idx_child[cls == 0 ? 3 : 2];
      DevNode na{}, nb{};
      na.env_slot = nb.env_slot = -1;
      na.leaf = nb.leaf = -1;
      if (ca >= 0) na = p.nodes[ca];
      if (cbx >= 0) nb = p.nodes[cbx];
      const double cfa = na.leaf >= 0 ? p.leaf_coef[na.leaf] : 0.0;
      const double cfb = nb.leaf >= 0 ? p.leaf_coef[nb.leaf] : 0.0;
      const cplx *bara = na.env_slot >= 0 ? p.bar_cur + ((size_t)b * p.maxslot + na.env_slot) * ENV_ELEMS : nullptr;
      const cplx *barb = nb.env_slot >= 0 ? p.bar_cur + ((size_t)b * p.maxslot + nb.env_slot) * ENV_ELEMS : nullptr;
      __syncwarp();   // the previous class's D is consumed
      for (int e = lane; e < ENV_ELEMS; e += 32) {
        const cplx rc = cconj(R[e]);
        cplx xa = cscale(rc, cfa), xb = cscale(rc, cfb);
        if (bara) xa = cadd(xa, bara[e]);
        if (barb) xb = cadd(xb, barb[e]);
        cplx d0, d1;
        if (cls == 0) {
          d0 = cadd(xa, xb);
          d1 = csub(xa, xb);
        } else {
          const cplx ixb = cmake(-xb.y, xb.x);
          d0 = cadd(xa, ixb);
          d1 = csub(xa, ixb);
        }
        D[(e >> 4) * MMA_S_STRIDE + (e & 15)] = d0;
        D[(CHI + (e >> 4)) * MMA_S_STRIDE + (e & 15)] = d1;
      }
      __syncwarp();
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        // output column tile ct covers panel half o = ct >> 1; operand source src(o)
        cplx af[2][2], df[4];
#pragma unroll
        for (int o = 0; o < 2; ++o) {
          const int src = cls == 0 ? o : 1 - o;
#pragma unroll
          for (int rt = 0; rt < 2; ++rt) af[o][rt] = A[(rt * 8 + g) * MMA_A_STRIDE + src * CHI + ks * 4 + t];
        }
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) {
          const int src = cls == 0 ? (ct >> 1) : 1 - (ct >> 1);
          df[ct] = D[(src * CHI + ks * 4 + t) * MMA_S_STRIDE + (ct & 1) * 8 + g];
        }
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 4; ++ct) {
            const cplx a = af[ct >> 1][rt], d = df[ct];
            dmma(yr[rt][ct][0], yr[rt][ct][1], a.x, d.x);
            dmma(yr[rt][ct][0], yr[rt][ct][1], -a.y, d.y);
            dmma(yi[rt][ct][0], yi[rt][ct][1], a.x, d.y);
            dmma(yi[rt][ct][0], yi[rt][ct][1], a.y, d.x);
          }
      }
    }
    // Y panel into the S region: Y_i[row][c] at S[(i * CHI + row) * MMA_S_STRIDE + c]
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 4; ++ct)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int col = ct * 8 + 2 * t + j;
          S[((col >> 4) * CHI + rt * 8 + g) * MMA_S_STRIDE + (col & 15)] = cmake(yr[rt][ct][j], yi[rt][ct][j]);
        }
    __syncwarp();
    // site cotangent: Abar_o += E Y_o (= S_src D_src summed over the classes, with S = E A)
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      cplx ef[2], yf[4];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt) ef[rt] = E[(rt * 8 + g) * MMA_E_STRIDE + ks * 4 + t];
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) yf[ct] = S[((ct >> 1) * CHI + ks * 4 + t) * MMA_S_STRIDE + (ct & 1) * 8 + g];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) {
          const cplx x = ef[rt], d = yf[ct];
          dmma(abr[rt][ct][0], abr[rt][ct][1], x.x, d.x);
          dmma(abr[rt][ct][0], abr[rt][ct][1], -x.y, d.y);
          dmma(abi[rt][ct][0], abi[rt][ct][1], x.x, d.y);
          dmma(abi[rt][ct][0], abi[rt][ct][1], x.y, d.x);
        }
    }
    __syncwarp();   // E is consumed: prefetch the next parent
    if (gidx + GLEVEL_WARPS < g1) grad_stage_parent(p, b, gidx + GLEVEL_WARPS, E, lane);
    cp_async_commit();
    if (p.s > 0) {
      // parent cotangent Ebar = sum_i Y_i A_i^H. Cotangents of Hermitian
      // environments are Hermitian: the tiles (0,0), (0,1), (1,1) are formed and
      // (1,0) is stored as the conjugate transpose of (0,1).
      double orr[2][2][2], oi[2][2][2];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 2; ++ct)
#pragma unroll
          for (int j = 0; j < 2; ++j) orr[rt][ct][j] = oi[rt][ct][j] = 0.0;
#pragma unroll
      for (int ks = 0; ks < 8; ++ks) {
        const int kk = ks * 4 + t;            // (i, k) = (kk >> 4, kk & 15)
        cplx yf[2], bf[2];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt) yf[rt] = S[((kk >> 4) * CHI + rt * 8 + g) * MMA_S_STRIDE + (kk & 15)];
#pragma unroll
        for (int ct = 0; ct < 2; ++ct) bf[ct] = A[(ct * 8 + g) * MMA_A_STRIDE + kk];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 2; ++ct) {
            if (rt == 1 && ct == 0) continue;
            // Y conj(A): re = Yr Ar + Yi Ai, im = Yi Ar - Yr Ai
            dmma(orr[rt][ct][0], orr[rt][ct][1], yf[rt].x, bf[ct].x);
            dmma(orr[rt][ct][0], orr[rt][ct][1], yf[rt].y, bf[ct].y);
            dmma(oi[rt][ct][0], oi[rt][ct][1], yf[rt].y, bf[ct].x);
            dmma(oi[rt][ct][0], oi[rt][ct][1], -yf[rt].x, bf[ct].y);
          }
      }
      cplx *dst = grp.parent_slot >= 0 ? p.bar_prev + ((size_t)b * p.maxslot + grp.parent_slot) * ENV_ELEMS
                                       : p.rootbar + ((size_t)b * p.n + p.s) * ENV_ELEMS;   // suffix root
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = rt; ct < 2; ++ct)
#pragma unroll
          for (int j = 0; j < 2; ++j)
            dst[(rt * 8 + g) * CHI + ct * 8 + 2 * t + j] = cmake(orr[rt][ct][j], oi[rt][ct][j]);
#pragma unroll
      for (int j = 0; j < 2; ++j) dst[(8 + 2 * t + j) * CHI + g] = cmake(orr[0][1][j], -oi[0][1][j]);
    }
    __syncwarp();   // S / D are rewritten by the next group
  }
  cp_async_wait<0>();
  __syncthreads();
  // fixed-order combination of the warps' site cotangent panels (times 2)
  cplx *panel = sm.S[warp];     // 576 >= 512 entries, one per site element
#pragma unroll
  for (int rt = 0; rt < 2; ++rt)
#pragma unroll
    for (int ct = 0; ct < 4; ++ct)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int col = ct * 8 + 2 * t + j;
        panel[((rt * 8 + g) * 2 + (col >> 4)) * CHI + (col & 15)] = cmake(2.0 * abr[rt][ct][j], 2.0 * abi[rt][ct][j]);
      }
  __syncthreads();
  cplx *dst = p.partial + ((size_t)b * gridDim.x + blockIdx.x) * SITE_ELEMS;
  for (int e = threadIdx.x; e < SITE_ELEMS; e += GLEVEL_WARPS * 32) {
    cplx acc = sm.S[0][e];
    for (int w = 1; w < GLEVEL_WARPS; ++w) acc = cadd(acc, sm.S[w][e]);
    dst[e] = acc;
  }
}

// ---------------------------------------------------------------------------
// backward level for a circuit of real gates. Its site tiles are real and its
// environments i^k Er: real for an even phase k, imaginary for an odd one. A
// word with an odd number of Y's has the value zero at every angle, and so has a
// pair closure of odd phase sum; their cotangents reach only the imaginary parts
// of the site cotangents, which a gradient with respect to real gate angles
// never reads. Left out (their leaf weights taken as zero here, odd pairs masked
// by split_pair_bwd_kernel), every cotangent is of its node's kind, like the
// environment, so D, Y = A D and the parent cotangent Y A^T are of the parent's
// kind (DevGroup::classes bit 2) and the site cotangent E Y is real: one real
// DMMA product where grad_bwd_level_mma_body issues four, on the same operands in
// the same order, so the real parts of the site cotangents -- and the angle
// gradients -- keep that kernel's bits. Shared memory holds only the nonzero
// parts (a double per element): 57 KB per CTA, three CTAs per SM, against
// 106 KB for the complex tiles.
// ---------------------------------------------------------------------------
constexpr int GR_A_STRIDE = 36;   // real site tile, rows [a] of [i * 16 + c]
constexpr int GR_E_STRIDE = 20;   // one part of the parent environment, 16 rows
constexpr int GR_S_STRIDE = 20;   // one part of a [2][16][16] panel (D, Y)

struct GradBwdRealSmem {
  double A[CHI * GR_A_STRIDE];
  double R[ENV_ELEMS];
  double E[GLEVEL_WARPS][CHI * GR_E_STRIDE];
  double S[GLEVEL_WARPS][2 * CHI * GR_S_STRIDE];   // Y panel; at the end the site cotangent panel
  double D[GLEVEL_WARPS][2 * CHI * GR_S_STRIDE];
};

// Hint: bring the 128-byte line at p into L2 (no effect on results).
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}

// The nonzero part of group grp's parent environment into E (cp.async): a
// parent of the previous level is stored as that part (ENV_ELEMS doubles; no
// cut level is a parent), the vacuum and a suffix root R_{s+1} are real.
__device__ __forceinline__ void grad_stage_parent_real(const GradLevelParams &p, int b, const DevGroup &grp, double *E,
                                                       int lane) {
  if (grp.parent_slot < 0 && !p.suffix) {
    for (int e = lane; e < ENV_ELEMS; e += 32) E[(e >> 4) * GR_E_STRIDE + (e & 15)] = e == 0 ? 1.0 : 0.0;
    return;
  }
  if (grp.parent_slot < 0) {
    const double *src = reinterpret_cast<const double *>(p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS);
    for (int e = lane; e < ENV_ELEMS; e += 32) cp_async8(E + (e >> 4) * GR_E_STRIDE + (e & 15), src + 2 * e);
    return;
  }
  const double *src =
      reinterpret_cast<const double *>(p.env_prev + (size_t)b * p.prev_stride + (size_t)grp.parent_slot * ENV_ELEMS);
  for (int e = 2 * lane; e < ENV_ELEMS; e += 64) cp_async16(E + (e >> 4) * GR_E_STRIDE + (e & 15), src + e);
}


__device__ __forceinline__ void grad_bwd_level_real_body(const GradLevelParams &p, unsigned char *smem_raw) {
  GradBwdRealSmem &sm = *reinterpret_cast<GradBwdRealSmem *>(smem_raw);
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {
    const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
    const cplx *rg = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
    for (int e = threadIdx.x; e < SITE_ELEMS; e += GLEVEL_WARPS * 32) sm.A[(e >> 5) * GR_A_STRIDE + (e & 31)] = ag[e].x;
    for (int e = threadIdx.x; e < ENV_ELEMS; e += GLEVEL_WARPS * 32) sm.R[e] = rg[e].x;
  }
  __syncthreads();
  const double *A = sm.A;
  const double *R = sm.R;
  double *E = sm.E[warp];
  double *S = sm.S[warp];
  double *D = sm.D[warp];
  const int g = lane >> 2, t = lane & 3;
  // site cotangent panel of this warp (real): rows rt * 8 + g, cols ct * 8 + 2t + j of [Abar_0 | Abar_1]
  double abr[2][4][2];
#pragma unroll
  for (int rt = 0; rt < 2; ++rt)
#pragma unroll
    for (int ct = 0; ct < 4; ++ct) abr[rt][ct][0] = abr[rt][ct][1] = 0.0;
  const int per_cta = GLEVEL_WARPS * GROUPS_PER_WARP;
  const int g0 = blockIdx.x * per_cta;
  const int g1 = min(g0 + per_cta, p.ngroups);
  int gidx = g0 + warp;
  // the next group's child records, one per lane (at most four), loaded when its
  // parent is staged and read back with shuffles
  DevNode nd_next{};
  if (gidx < g1) {
    const DevGroup gf = p.groups[gidx];
    grad_stage_parent_real(p, b, gf, E, lane);
    if (lane < gf.nchild) nd_next = p.nodes[gf.child_begin + lane];
    cp_async_commit();
  }
  auto shfl_node = [&](const DevNode &v, int src) {
    DevNode r;
    r.code = __shfl_sync(0xffffffffu, v.code, src);
    r.env_slot = __shfl_sync(0xffffffffu, v.env_slot, src);
    r.leaf = __shfl_sync(0xffffffffu, v.leaf, src);
    r.phase = __shfl_sync(0xffffffffu, v.phase, src);
    return r;
  };
  for (; gidx < g1; gidx += GLEVEL_WARPS) {
    cp_async_wait<0>();
    __syncwarp();
    const DevGroup grp = p.groups[gidx];
    const bool odd = (grp.classes & 4) != 0;
    const DevNode nd = nd_next;
    int idx_child[4] = {-1, -1, -1, -1};   // child (lane of nd) of each Pauli code
    for (int ci = 0; ci < grp.nchild; ++ci) idx_child[__shfl_sync(0xffffffffu, nd.code, ci)] = ci;
    // Y_o = sum over classes of A_src(o) D_src(o), one part
    double yr[2][4][2];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) yr[rt][ct][0] = yr[rt][ct][1] = 0.0;
    for (int cls = 0; cls < 2; ++cls) {
      if (!(grp.classes & (1 << cls))) continue;
      const int ca = idx_child[cls == 0 ? 0 : 1], cbx = idx_child[cls == 0 ? 3 : 2];
      DevNode na{}, nb{};
      na.env_slot = nb.env_slot = -1;
      na.leaf = nb.leaf = -1;
      const DevNode ra = shfl_node(nd, ca < 0 ? 0 : ca), rb = shfl_node(nd, cbx < 0 ? 0 : cbx);
      if (ca >= 0) na = ra;
      if (cbx >= 0) nb = rb;
      // leaves of odd phase are left out (zero value at every angle)
      const double cfa = na.leaf >= 0 && !(na.phase & 1) ? p.leaf_coef[na.leaf] : 0.0;
      const double cfb = nb.leaf >= 0 && !(nb.phase & 1) ? p.leaf_coef[nb.leaf] : 0.0;
      const cplx *bara = na.env_slot >= 0 ? p.bar_cur + ((size_t)b * p.maxslot + na.env_slot) * ENV_ELEMS : nullptr;
      const cplx *barb = nb.env_slot >= 0 ? p.bar_cur + ((size_t)b * p.maxslot + nb.env_slot) * ENV_ELEMS : nullptr;
      __syncwarp();   // the previous class's D is consumed
      for (int e = lane; e < ENV_ELEMS; e += 32) {
        // the complex D entries of the four-product kernels, of which the part of
        // the parent's kind is kept (the other is zero)
        const cplx rc = cmake(R[e], -0.0);
        cplx xa = cscale(rc, cfa), xb = cscale(rc, cfb);
        if (bara) xa = cadd(xa, bara[e]);
        if (barb) xb = cadd(xb, barb[e]);
        cplx d0, d1;
        if (cls == 0) {
          d0 = cadd(xa, xb);
          d1 = csub(xa, xb);
        } else {
          const cplx ixb = cmake(-xb.y, xb.x);
          d0 = cadd(xa, ixb);
          d1 = csub(xa, ixb);
        }
        D[(e >> 4) * GR_S_STRIDE + (e & 15)] = odd ? d0.y : d0.x;
        D[(CHI + (e >> 4)) * GR_S_STRIDE + (e & 15)] = odd ? d1.y : d1.x;
      }
      __syncwarp();
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        double af[2][2], df[4];
#pragma unroll
        for (int o = 0; o < 2; ++o) {
          const int src = cls == 0 ? o : 1 - o;
#pragma unroll
          for (int rt = 0; rt < 2; ++rt) af[o][rt] = A[(rt * 8 + g) * GR_A_STRIDE + src * CHI + ks * 4 + t];
        }
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) {
          const int src = cls == 0 ? (ct >> 1) : 1 - (ct >> 1);
          df[ct] = D[(src * CHI + ks * 4 + t) * GR_S_STRIDE + (ct & 1) * 8 + g];
        }
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 4; ++ct) dmma(yr[rt][ct][0], yr[rt][ct][1], af[ct >> 1][rt], df[ct]);
      }
    }
    // Y panel (one part) into S: Y_i[row][c] at S[(i * CHI + row) * GR_S_STRIDE + c]
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 4; ++ct)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int col = ct * 8 + 2 * t + j;
          S[((col >> 4) * CHI + rt * 8 + g) * GR_S_STRIDE + (col & 15)] = yr[rt][ct][j];
        }
    __syncwarp();
    // site cotangent (real): even Abar += Er Yr, odd Abar += -Ei Yi
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      double ef[2], yf[4];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt) {
        const double x = E[(rt * 8 + g) * GR_E_STRIDE + ks * 4 + t];
        ef[rt] = odd ? -x : x;
      }
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) yf[ct] = S[((ct >> 1) * CHI + ks * 4 + t) * GR_S_STRIDE + (ct & 1) * 8 + g];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) dmma(abr[rt][ct][0], abr[rt][ct][1], ef[rt], yf[ct]);
    }
    __syncwarp();   // E is consumed: prefetch the next parent
    // and its child records; the cotangents of its children (lanes 8c .. 8c + 7:
    // child c) are warmed into L2 below, after the parent cotangent product
    const bool has_next = gidx + GLEVEL_WARPS < g1;
    int next_nchild = 0;
    if (has_next) {
      const DevGroup gn = p.groups[gidx + GLEVEL_WARPS];
      grad_stage_parent_real(p, b, gn, E, lane);
      next_nchild = gn.nchild;
      nd_next = DevNode{};
      if (lane < gn.nchild) nd_next = p.nodes[gn.child_begin + lane];
    }
    cp_async_commit();
    if (p.s > 0) {
      // parent cotangent Ebar = sum_i Y_i A_i^T, tiles (0,0), (0,1), (1,1); the
      // (1,0) tile is the conjugate transpose of (0,1)
      double o[2][2][2];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 2; ++ct) o[rt][ct][0] = o[rt][ct][1] = 0.0;
#pragma unroll
      for (int ks = 0; ks < 8; ++ks) {
        const int kk = ks * 4 + t;            // (i, k) = (kk >> 4, kk & 15)
        double yf[2], bf[2];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt) yf[rt] = S[((kk >> 4) * CHI + rt * 8 + g) * GR_S_STRIDE + (kk & 15)];
#pragma unroll
        for (int ct = 0; ct < 2; ++ct) bf[ct] = A[(ct * 8 + g) * GR_A_STRIDE + kk];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 2; ++ct) {
            if (rt == 1 && ct == 0) continue;
            dmma(o[rt][ct][0], o[rt][ct][1], yf[rt], bf[ct]);
          }
      }
      cplx *dst = grp.parent_slot >= 0 ? p.bar_prev + ((size_t)b * p.maxslot + grp.parent_slot) * ENV_ELEMS
                                       : p.rootbar + ((size_t)b * p.n + p.s) * ENV_ELEMS;   // suffix root
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = rt; ct < 2; ++ct)
#pragma unroll
          for (int j = 0; j < 2; ++j)
            dst[(rt * 8 + g) * CHI + ct * 8 + 2 * t + j] = odd ? cmake(0.0, o[rt][ct][j]) : cmake(o[rt][ct][j], 0.0);
#pragma unroll
      for (int j = 0; j < 2; ++j)
        dst[(8 + 2 * t + j) * CHI + g] = odd ? cmake(0.0, -o[0][1][j]) : cmake(o[0][1][j], -0.0);
    }
    int next_slot = -1;
    if (has_next) {
      const int sl = __shfl_sync(0xffffffffu, nd_next.env_slot, lane >> 3);
      if ((lane >> 3) < next_nchild) next_slot = sl;
    }
    if (next_slot >= 0) {   // 4 KB cotangent = 32 lines, four per lane of the child's eight
      const char *line = reinterpret_cast<const char *>(p.bar_cur + ((size_t)b * p.maxslot + next_slot) * ENV_ELEMS);
#pragma unroll
      for (int l = 0; l < 4; ++l) prefetch_l2(line + ((lane & 7) * 4 + l) * 128);
    }
    __syncwarp();   // S / D are rewritten by the next group
  }
  cp_async_wait<0>();
  __syncthreads();
  // fixed-order combination of the warps' site cotangent panels (times 2)
  double *panel = sm.S[warp];     // 640 >= 512 entries, one per site element
#pragma unroll
  for (int rt = 0; rt < 2; ++rt)
#pragma unroll
    for (int ct = 0; ct < 4; ++ct)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int col = ct * 8 + 2 * t + j;
        panel[((rt * 8 + g) * 2 + (col >> 4)) * CHI + (col & 15)] = 2.0 * abr[rt][ct][j];
      }
  __syncthreads();
  cplx *dst = p.partial + ((size_t)b * gridDim.x + blockIdx.x) * SITE_ELEMS;
  for (int e = threadIdx.x; e < SITE_ELEMS; e += GLEVEL_WARPS * 32) {
    double acc = sm.S[0][e];
    for (int w = 1; w < GLEVEL_WARPS; ++w) acc += sm.S[w][e];
    dst[e] = cmake(acc, 0.0);
  }
}

// ---------------------------------------------------------------------------
// forward level for a circuit of real gates on one-part shared tiles: the
// products of grad_fwd_level_mma_body<0> without the exact-zero terms of the
// real site tile and of E's zero part (E and S = E A are of the parent's kind,
// DevGroup::classes bit 2: one real DMMA product per complex one), only the
// nonzero parts of E and S in shared memory, and the children's complex values
// and leaf sums formed by the same expressions (same bits). 55 KB per CTA
// against 85 KB.
// ---------------------------------------------------------------------------
struct GradFwdRealSmem {
  double A[CHI * GR_A_STRIDE];
  cplx R[ENV_ELEMS];
  double E[GLEVEL_WARPS][CHI * GR_E_STRIDE];
  double S[GLEVEL_WARPS][2 * CHI * GR_S_STRIDE];
  cplx L[GLEVEL_WARPS][ENV_ELEMS];
};

__device__ __forceinline__ void grad_fwd_level_real_body(const GradLevelParams &p, unsigned char *smem_raw) {
  GradFwdRealSmem &sm = *reinterpret_cast<GradFwdRealSmem *>(smem_raw);
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {
    const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
    const cplx *rg = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
    for (int e = threadIdx.x; e < SITE_ELEMS; e += GLEVEL_WARPS * 32) sm.A[(e >> 5) * GR_A_STRIDE + (e & 31)] = ag[e].x;
    for (int e = threadIdx.x; e < ENV_ELEMS; e += GLEVEL_WARPS * 32) sm.R[e] = rg[e];
    for (int e = lane; e < ENV_ELEMS; e += 32) sm.L[warp][e] = cmake(0, 0);
  }
  __syncthreads();
  const double *A = sm.A;
  const cplx *R = sm.R;
  double *E = sm.E[warp];
  double *S = sm.S[warp];
  cplx *L = sm.L[warp];
  const int g = lane >> 2, t = lane & 3;
  const int per_cta = GLEVEL_WARPS * GROUPS_PER_WARP;
  const int g0 = blockIdx.x * per_cta;
  const int g1 = min(g0 + per_cta, p.ngroups);
  int gidx = g0 + warp;
  if (gidx < g1) {
    grad_stage_parent_real(p, b, p.groups[gidx], E, lane);
    cp_async_commit();
  }
  for (; gidx < g1; gidx += GLEVEL_WARPS) {
    cp_async_wait<0>();
    __syncwarp();
    const DevGroup grp = p.groups[gidx];
    const bool odd = (grp.classes & 4) != 0;
    // the children's node records, one per lane (at most four), loaded while the
    // S product runs and read back with shuffles
    DevNode nd{};
    if (lane < grp.nchild) nd = p.nodes[grp.child_begin + lane];
    // S = E [A_0 | A_1], one part
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
        for (int rt = 0; rt < 2; ++rt) ef[rt] = E[(rt * 8 + g) * GR_E_STRIDE + ks * 4 + t];
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) pf[ct] = A[(ks * 4 + t) * GR_A_STRIDE + ct * 8 + g];
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
            S[((col >> 4) * CHI + rt * 8 + g) * GR_S_STRIDE + (col & 15)] = sacc[rt][ct][j];
          }
    }
    __syncwarp();   // E is dead and S complete: prefetch the next parent
    if (gidx + GLEVEL_WARPS < g1) grad_stage_parent_real(p, b, p.groups[gidx + GLEVEL_WARPS], E, lane);
    cp_async_commit();
    for (int cls = 0; cls < 2; ++cls) {
      if (!(grp.classes & (1 << cls))) continue;
      // one part of t0 = A_x^H S_y (and of t1): I/Z t0 = A_0^T S_0, t1 = A_1^T S_1
      // over tiles (0,0), (0,1), (1,1); X/Y t0 = A_0^T S_1 over four tiles and
      // t1 = t0^H through the panel
      double a[2][2][2], c[2][2][2];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 2; ++ct) a[rt][ct][0] = a[rt][ct][1] = c[rt][ct][0] = c[rt][ct][1] = 0.0;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        double x0[2], x1[2], y0[2], y1[2];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt) {
          x0[rt] = A[(ks * 4 + t) * GR_A_STRIDE + rt * 8 + g];
          x1[rt] = A[(ks * 4 + t) * GR_A_STRIDE + CHI + rt * 8 + g];
        }
#pragma unroll
        for (int ct = 0; ct < 2; ++ct) {
          y0[ct] = S[(ks * 4 + t) * GR_S_STRIDE + ct * 8 + g];
          y1[ct] = S[(CHI + ks * 4 + t) * GR_S_STRIDE + ct * 8 + g];
        }
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 2; ++ct) {
            if (cls == 0) {
              if (rt == 1 && ct == 0) continue;
              dmma(a[rt][ct][0], a[rt][ct][1], x0[rt], y0[ct]);
              dmma(c[rt][ct][0], c[rt][ct][1], x1[rt], y1[ct]);
            } else {
              dmma(a[rt][ct][0], a[rt][ct][1], x0[rt], y1[ct]);
            }
          }
      }
      if (cls == 1) {
        __syncwarp();   // the panel is consumed: t0 goes into its place
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) S[(rt * 8 + g) * GR_S_STRIDE + ct * 8 + 2 * t + j] = a[rt][ct][j];
        __syncwarp();
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = rt; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) c[rt][ct][j] = S[(ct * 8 + 2 * t + j) * GR_S_STRIDE + rt * 8 + g];
      }
      for (int ci = 0; ci < grp.nchild; ++ci) {
        DevNode node;
        node.code = __shfl_sync(0xffffffffu, nd.code, ci);
        node.env_slot = __shfl_sync(0xffffffffu, nd.env_slot, ci);
        node.leaf = __shfl_sync(0xffffffffu, nd.leaf, ci);
        node.phase = __shfl_sync(0xffffffffu, nd.phase, ci);
        const bool iz = (node.code == 0 || node.code == 3);
        if (iz != (cls == 0)) continue;
        cplx out[2][2][2];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = rt; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              // the complex t0, t1 of the four-product kernels (zero part exact)
              const double pa = a[rt][ct][j], pc = c[rt][ct][j];
              const cplx t0 = odd ? cmake(0.0, pa) : cmake(pa, 0.0);
              const cplx t1 = cls == 0 ? (odd ? cmake(0.0, pc) : cmake(pc, 0.0))
                                       : (odd ? cmake(0.0, -pc) : cmake(pc, -0.0));
              if (node.code == 0 || node.code == 1) out[rt][ct][j] = cadd(t0, t1);
              else if (node.code == 3) out[rt][ct][j] = csub(t0, t1);
              else { const cplx d = csub(t1, t0); out[rt][ct][j] = cmake(-d.y, d.x); }
            }
        // out[1][0][j]: the (1,0)-tile element this lane owns, [8 + 2t + j][g]
        out[1][0][0] = cconj(out[0][1][0]);
        out[1][0][1] = cconj(out[0][1][1]);
        if (node.env_slot >= 0) {
          cplx *dst = p.env_cur + (size_t)b * p.cur_stride + (size_t)node.env_slot * ENV_ELEMS;
          if (p.env_complex) {
#pragma unroll
            for (int rt = 0; rt < 2; ++rt)
#pragma unroll
              for (int ct = rt; ct < 2; ++ct)
#pragma unroll
                for (int j = 0; j < 2; ++j) dst[(rt * 8 + g) * CHI + ct * 8 + 2 * t + j] = out[rt][ct][j];
#pragma unroll
            for (int j = 0; j < 2; ++j) dst[(8 + 2 * t + j) * CHI + g] = out[1][0][j];
          } else {   // the nonzero part (the child's kind)
            double *dd = reinterpret_cast<double *>(dst);
            const bool oc = (node.phase & 1) != 0;
#pragma unroll
            for (int rt = 0; rt < 2; ++rt)
#pragma unroll
              for (int ct = rt; ct < 2; ++ct)
                *reinterpret_cast<double2 *>(dd + (rt * 8 + g) * CHI + ct * 8 + 2 * t) =
                    oc ? make_double2(out[rt][ct][0].y, out[rt][ct][1].y)
                       : make_double2(out[rt][ct][0].x, out[rt][ct][1].x);
#pragma unroll
            for (int j = 0; j < 2; ++j) dd[(8 + 2 * t + j) * CHI + g] = oc ? out[1][0][j].y : out[1][0][j].x;
          }
        }
        if (node.leaf >= 0 && p.leaf_work) {
          const double cf = p.leaf_coef[node.leaf];
          double v = 0.0;
#pragma unroll
          for (int rt = 0; rt < 2; ++rt)
#pragma unroll
            for (int ct = rt; ct < 2; ++ct)
#pragma unroll
              for (int j = 0; j < 2; ++j) {
                const int idx = (rt * 8 + g) * CHI + ct * 8 + 2 * t + j;
                const cplx rv = R[idx];
                v += out[rt][ct][j].x * rv.x - out[rt][ct][j].y * rv.y;
                L[idx] = cadd(L[idx], cscale(out[rt][ct][j], cf));
              }
#pragma unroll
          for (int j = 0; j < 2; ++j) {   // the (1,0) tile
            const int idx = (8 + 2 * t + j) * CHI + g;
            const cplx rv = R[idx];
            v += out[1][0][j].x * rv.x - out[1][0][j].y * rv.y;
            L[idx] = cadd(L[idx], cscale(out[1][0][j], cf));
          }
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) p.leafval[(size_t)b * p.nleaf + node.leaf] = v;
        }
      }
    }
    __syncwarp();   // S is rewritten by the next parent
  }
  cp_async_wait<0>();
  __syncthreads();
  if (!p.leaf_work) return;
  cplx *dst = p.partial + ((size_t)b * gridDim.x + blockIdx.x) * ENV_ELEMS;
  for (int e = threadIdx.x; e < ENV_ELEMS; e += GLEVEL_WARPS * 32) {
    cplx acc = sm.L[0][e];
    for (int w = 1; w < GLEVEL_WARPS; ++w) acc = cadd(acc, sm.L[w][e]);
    dst[e] = acc;
  }
}

// Forward gradient level for a circuit of real gates: real site tiles and
// environments i^k Er, one real product per complex one where the four-product
// kernel issues four (its bits); one-part shared tiles, three CTAs per SM.
__global__ void __launch_bounds__(GLEVEL_WARPS * 32, 3)
grad_fwd_level_real_a_kernel(GradLevelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  grad_fwd_level_real_body(p, smem_raw);
}

__global__ void __launch_bounds__(GLEVEL_WARPS * 32, 2)
grad_bwd_level_mma_kernel(GradLevelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  grad_bwd_level_mma_body(p, smem_raw);
}

// Backward gradient level for a circuit of real gates (real site tiles,
// one-part shared tiles; three CTAs per SM).
__global__ void __launch_bounds__(GLEVEL_WARPS * 32, 3)
grad_bwd_level_real_a_kernel(GradLevelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  grad_bwd_level_real_body(p, smem_raw);
}

}  // namespace vqemps
