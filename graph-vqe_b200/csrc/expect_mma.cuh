// Trie level on the FP64 tensor cores (DMMA, mma.sync m8n8k4 .f64).
//
// Same work and output as level_kernel (expect.cuh): one warp per trie parent,
// S_i = E A_i, then one product per Pauli class present among the children.
// Complex 16 x 16 products are four real DMMA products each:
//   Re(X Y) = Xr Yr - Xi Yi,  Im(X Y) = Xr Yi + Xi Yr,
// over 8 x 8 output tiles and k-steps of 4. A fragment element and its
// imaginary part are one 16-byte (re, im) load, so a k-step of the first half
// issues 6 shared loads per lane for 32 DMMAs (the SIMT kernel issues 8 loads
// per 16 complex FMAs). Shared tiles are padded so that every quarter-warp
// fragment load touches 32 distinct banks:
//   E:  16 rows, stride 20 complex (rows 0/1 of a quarter-warp 64 bytes apart mod 128)
//   A:  16 rows [a][i*16+c], stride 34 complex (4 rows 32 bytes apart mod 128)
//   S:  2 x 16 rows [i][a][c], stride 18 complex (4 rows 32 bytes apart mod 128)
// Fragment layout of m8n8k4 .f64 (PTX ISA): A (8x4 row): row = lane>>2,
// col = lane&3; B (4x8 col): row = lane&3, col = lane>>2; C/D (8x8): row = lane>>2,
// cols 2*(lane&3) + {0,1}.
#pragma once
#include "common.cuh"
#include "expect.cuh"

namespace vqemps {

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

constexpr int MMA_E_STRIDE = 20;
constexpr int MMA_A_STRIDE = 34;
constexpr int MMA_S_STRIDE = 18;

template <int WARPS>
struct LevelMmaSmem {
  cplx A[CHI * MMA_A_STRIDE];
  cplx W[WARPS][2 * CHI * MMA_S_STRIDE];   // per warp: padded E, then padded S_0 | S_1
};

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
level_mma_kernel(LevelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  LevelMmaSmem<WARPS> &sm = *reinterpret_cast<LevelMmaSmem<WARPS> *>(smem_raw);
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {
    const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
    for (int e = threadIdx.x; e < SITE_ELEMS; e += WARPS * 32)
      sm.A[(e >> 5) * MMA_A_STRIDE + (e & 31)] = ag[e];
  }
  __syncthreads();
  const int gidx = blockIdx.x * WARPS + warp;
  if (gidx >= p.ngroups) return;
  const DevGroup grp = p.groups[gidx];
  cplx *E = sm.W[warp];
  cplx *S = sm.W[warp];
  const cplx *A = sm.A;
  const int g = lane >> 2, t = lane & 3;

  if (grp.parent_slot < 0) {
    for (int e = lane; e < ENV_ELEMS; e += 32)
      E[(e >> 4) * MMA_E_STRIDE + (e & 15)] = cmake(e == 0 ? 1.0 : 0.0, 0.0);
  } else {
    const cplx *src = p.env_prev + ((size_t)b * p.nslot_prev + grp.parent_slot) * ENV_ELEMS;
    for (int e = lane; e < ENV_ELEMS; e += 32) E[(e >> 4) * MMA_E_STRIDE + (e & 15)] = src[e];
  }
  __syncwarp();

  // ---- first half: [S_0 | S_1] (16 x 32) = E (16 x 16) [A_0 | A_1] (16 x 32)
  {
    double sr[2][4][2], si[2][4][2];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 4; ++ct) { sr[rt][ct][0] = sr[rt][ct][1] = 0.0; si[rt][ct][0] = si[rt][ct][1] = 0.0; }
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
          dmma(sr[rt][ct][0], sr[rt][ct][1], er, pf[ct].x);
          dmma(sr[rt][ct][0], sr[rt][ct][1], nei, pf[ct].y);
          dmma(si[rt][ct][0], si[rt][ct][1], er, pf[ct].y);
          dmma(si[rt][ct][0], si[rt][ct][1], ei, pf[ct].x);
        }
      }
    }
    __syncwarp();   // every lane has read E before S overwrites it
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 4; ++ct)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int col = ct * 8 + 2 * t + j;          // panel column = i * 16 + c
          S[((col >> 4) * CHI + rt * 8 + g) * MMA_S_STRIDE + (col & 15)] = cmake(sr[rt][ct][j], si[rt][ct][j]);
        }
  }
  __syncwarp();

  // ---- second half: per class, tx = A_x^H S_y over the 16 x 16 output
  const cplx *R = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
  for (int cls = 0; cls < 2; ++cls) {
    if (!(grp.classes & (1 << cls))) continue;
    // cls 0: t0 = A_0^H S_0, t1 = A_1^H S_1 ; cls 1: t0 = A_0^H S_1 (u01), t1 = A_1^H S_0 (u10)
    const int y0 = cls == 0 ? 0 : 1, y1 = cls == 0 ? 1 : 0;
    double ar[2][2][2], ai[2][2][2], br[2][2][2], bi[2][2][2];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 2; ++ct)
#pragma unroll
        for (int j = 0; j < 2; ++j) ar[rt][ct][j] = ai[rt][ct][j] = br[rt][ct][j] = bi[rt][ct][j] = 0.0;
#pragma unroll
    for (int ks = 0; ks < 4; ++ks) {
      cplx a0[2], a1[2], s0[2], s1[2];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt) {
        a0[rt] = A[(ks * 4 + t) * MMA_A_STRIDE + rt * 8 + g];
        a1[rt] = A[(ks * 4 + t) * MMA_A_STRIDE + CHI + rt * 8 + g];
      }
#pragma unroll
      for (int ct = 0; ct < 2; ++ct) {
        s0[ct] = S[(y0 * CHI + ks * 4 + t) * MMA_S_STRIDE + ct * 8 + g];
        s1[ct] = S[(y1 * CHI + ks * 4 + t) * MMA_S_STRIDE + ct * 8 + g];
      }
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 2; ++ct) {
          // conj(A)^T S: re = Ar Sr + Ai Si, im = Ar Si - Ai Sr
          dmma(ar[rt][ct][0], ar[rt][ct][1], a0[rt].x, s0[ct].x);
          dmma(ar[rt][ct][0], ar[rt][ct][1], a0[rt].y, s0[ct].y);
          dmma(ai[rt][ct][0], ai[rt][ct][1], a0[rt].x, s0[ct].y);
          dmma(ai[rt][ct][0], ai[rt][ct][1], -a0[rt].y, s0[ct].x);
          dmma(br[rt][ct][0], br[rt][ct][1], a1[rt].x, s1[ct].x);
          dmma(br[rt][ct][0], br[rt][ct][1], a1[rt].y, s1[ct].y);
          dmma(bi[rt][ct][0], bi[rt][ct][1], a1[rt].x, s1[ct].y);
          dmma(bi[rt][ct][0], bi[rt][ct][1], -a1[rt].y, s1[ct].x);
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
        for (int ct = 0; ct < 2; ++ct)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const cplx t0 = cmake(ar[rt][ct][j], ai[rt][ct][j]);
            const cplx t1 = cmake(br[rt][ct][j], bi[rt][ct][j]);
            if (node.code == 0 || node.code == 1) out[rt][ct][j] = cadd(t0, t1);
            else if (node.code == 3) out[rt][ct][j] = csub(t0, t1);
            else { const cplx d = csub(t1, t0); out[rt][ct][j] = cmake(-d.y, d.x); }   // Y
          }
      if (node.env_slot >= 0) {
        cplx *dst = p.env_cur + ((size_t)b * p.nslot_cur + node.env_slot) * ENV_ELEMS;
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) dst[(rt * 8 + g) * CHI + ct * 8 + 2 * t + j] = out[rt][ct][j];
      }
      if (node.leaf >= 0) {
        double v = 0.0;
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int ct = 0; ct < 2; ++ct)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
              const cplx rv = R[(rt * 8 + g) * CHI + ct * 8 + 2 * t + j];
              v += out[rt][ct][j].x * rv.x - out[rt][ct][j].y * rv.y;
            }
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) p.leafval[(size_t)b * p.nleaf_total + node.leaf] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// DMMA with persistent warps and parent prefetch (cp.async), R staged per CTA:
// the arithmetic of level_mma_kernel with the pipeline of level_pf_kernel. A
// warp owns a padded 5 KiB parent slot and a padded 9 KiB S panel; the next
// parent is copied into the slot as soon as the first half is done.
// ---------------------------------------------------------------------------
constexpr int MPF_WARPS = 4;

struct LevelMmaPfSmem {
  cplx A[CHI * MMA_A_STRIDE];
  cplx R[ENV_ELEMS];
  cplx E[MPF_WARPS][CHI * MMA_E_STRIDE];
  cplx S[MPF_WARPS][2 * CHI * MMA_S_STRIDE];
};

__device__ __forceinline__ void stage_parent_padded(const LevelParams &p, int b, int g, cplx *E, int lane) {
  const DevGroup grp = p.groups[g];
  if (grp.parent_slot < 0 && p.suffix) {
    const cplx *src = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
    for (int e = lane; e < ENV_ELEMS; e += 32) cp_async16(E + (e >> 4) * MMA_E_STRIDE + (e & 15), src + e);
  } else if (grp.parent_slot < 0) {
    for (int e = lane; e < ENV_ELEMS; e += 32)
      E[(e >> 4) * MMA_E_STRIDE + (e & 15)] = cmake(e == 0 ? 1.0 : 0.0, 0.0);
  } else {
    const cplx *src = p.env_prev + ((size_t)b * p.nslot_prev + grp.parent_slot) * ENV_ELEMS;
    for (int e = lane; e < ENV_ELEMS; e += 32) cp_async16(E + (e >> 4) * MMA_E_STRIDE + (e & 15), src + e);
  }
}

// Class-product tiles of conj(A_x)^T S_y (x = column offset 0 or CHI of the A
// panel, y = panel half) over the 8 x 8 output tiles (rt, ct); SKIP10 leaves
// the (1,0) tile out. KIND 1 (Gauss): k1 = Yr (Xr - Xi), k2 = Xr (Yi - Yr),
// k3 = -Xi (Yr + Yi), Re = k1 - k3, Im = k1 + k2; KIND 0: four real products.
template <int KIND, bool SKIP10>
__device__ __forceinline__ void class_tiles(const cplx *A, int xoff, const cplx *S, int y, double (&re)[2][2][2],
                                            double (&im)[2][2][2], int g, int t) {
  double k3[2][2][2];
#pragma unroll
  for (int rt = 0; rt < 2; ++rt)
#pragma unroll
    for (int ct = 0; ct < 2; ++ct)
#pragma unroll
      for (int j = 0; j < 2; ++j) re[rt][ct][j] = im[rt][ct][j] = k3[rt][ct][j] = 0.0;
#pragma unroll
  for (int ks = 0; ks < 4; ++ks) {
    cplx x[2], yv[2];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt) x[rt] = A[(ks * 4 + t) * MMA_A_STRIDE + xoff + rt * 8 + g];
#pragma unroll
    for (int ct = 0; ct < 2; ++ct) yv[ct] = S[(y * CHI + ks * 4 + t) * MMA_S_STRIDE + ct * 8 + g];
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 2; ++ct) {
        if (SKIP10 && rt == 1 && ct == 0) continue;
        if constexpr (KIND == 1) {
          dmma(re[rt][ct][0], re[rt][ct][1], x[rt].x - x[rt].y, yv[ct].x);
          dmma(im[rt][ct][0], im[rt][ct][1], x[rt].x, yv[ct].y - yv[ct].x);
          dmma(k3[rt][ct][0], k3[rt][ct][1], -x[rt].y, yv[ct].x + yv[ct].y);
        } else {
          dmma(re[rt][ct][0], re[rt][ct][1], x[rt].x, yv[ct].x);
          dmma(re[rt][ct][0], re[rt][ct][1], x[rt].y, yv[ct].y);
          dmma(im[rt][ct][0], im[rt][ct][1], x[rt].x, yv[ct].y);
          dmma(im[rt][ct][0], im[rt][ct][1], -x[rt].y, yv[ct].x);
        }
      }
  }
  if constexpr (KIND == 1) {
#pragma unroll
    for (int rt = 0; rt < 2; ++rt)
#pragma unroll
      for (int ct = 0; ct < 2; ++ct)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const double k1 = re[rt][ct][j];
          re[rt][ct][j] = k1 - k3[rt][ct][j];
          im[rt][ct][j] = k1 + im[rt][ct][j];
        }
  }
}

// GAUSS selects the complex product: false = four real DMMA products
// (Re = XrYr - XiYi, Im = XrYi + XiYr); true = Gauss's three-product form
// k1 = Yr (Xr + Xi), k2 = Xr (Yi - Yr), k3 = Xi (Yr + Yi), Re = k1 - k3,
// Im = k1 + k2, which trades a quarter of the tensor-pipe work for operand sums
// on the FMA pipe and a third accumulator.
template <bool GAUSS>
__device__ __forceinline__ void level_mma_pf_body(const LevelParams &p, int groups_per_warp,
                                                  unsigned char *smem_raw) {
  LevelMmaPfSmem &sm = *reinterpret_cast<LevelMmaPfSmem *>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // uniform batch: state blockIdx.y, groups interleaved over the grid;
  // work list: state w[0], groups w[1] .. w[1] + w[2] split over the warps
  int b, stride, first, count = 0;
  if (p.work != nullptr) {
    const int32_t *w = p.work + 3 * blockIdx.x;
    b = w[0];
    stride = MPF_WARPS;
    first = w[1] + warp;
    if (warp < w[2]) count = (w[2] - warp + MPF_WARPS - 1) / MPF_WARPS;
  } else {
    b = blockIdx.y;
    stride = gridDim.x * MPF_WARPS;
    first = blockIdx.x * MPF_WARPS + warp;
    if (first < p.ngroups) count = min(groups_per_warp, (p.ngroups - first + stride - 1) / stride);
  }
  {
    const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
    const cplx *rg = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
    for (int e = threadIdx.x; e < SITE_ELEMS; e += MPF_WARPS * 32) sm.A[(e >> 5) * MMA_A_STRIDE + (e & 31)] = ag[e];
    for (int e = threadIdx.x; e < ENV_ELEMS; e += MPF_WARPS * 32) sm.R[e] = rg[e];
  }
  __syncthreads();
  const cplx *A = sm.A;
  const cplx *R = sm.R;
  cplx *E = sm.E[warp];
  cplx *S = sm.S[warp];
  const int g = lane >> 2, t = lane & 3;
  if (count == 0) return;
  stage_parent_padded(p, b, first, E, lane);
  cp_async_commit();
  for (int k = 0; k < count; ++k) {
    const int gidx = first + k * stride;
    cp_async_wait<0>();
    __syncwarp();
    const DevGroup grp = p.groups[gidx];
    if constexpr (!GAUSS) {
      double sr[2][4][2], si[2][4][2];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) { sr[rt][ct][0] = sr[rt][ct][1] = 0.0; si[rt][ct][0] = si[rt][ct][1] = 0.0; }
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
            dmma(sr[rt][ct][0], sr[rt][ct][1], er, pf[ct].x);
            dmma(sr[rt][ct][0], sr[rt][ct][1], nei, pf[ct].y);
            dmma(si[rt][ct][0], si[rt][ct][1], er, pf[ct].y);
            dmma(si[rt][ct][0], si[rt][ct][1], ei, pf[ct].x);
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
            S[((col >> 4) * CHI + rt * 8 + g) * MMA_S_STRIDE + (col & 15)] = cmake(sr[rt][ct][j], si[rt][ct][j]);
          }
    } else {
      // S = E A with X = E (row operand), Y = A (column operand)
      double k1[2][4][2], k2[2][4][2], k3[2][4][2];
#pragma unroll
      for (int rt = 0; rt < 2; ++rt)
#pragma unroll
        for (int ct = 0; ct < 4; ++ct)
#pragma unroll
          for (int j = 0; j < 2; ++j) k1[rt][ct][j] = k2[rt][ct][j] = k3[rt][ct][j] = 0.0;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        cplx ef[2], pf[4];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt) ef[rt] = E[(rt * 8 + g) * MMA_E_STRIDE + ks * 4 + t];
#pragma unroll
        for (int ct = 0; ct < 4; ++ct) pf[ct] = A[(ks * 4 + t) * MMA_A_STRIDE + ct * 8 + g];
#pragma unroll
        for (int rt = 0; rt < 2; ++rt) {
          const double xs = ef[rt].x + ef[rt].y;
#pragma unroll
          for (int ct = 0; ct < 4; ++ct) {
            dmma(k1[rt][ct][0], k1[rt][ct][1], xs, pf[ct].x);
            dmma(k2[rt][ct][0], k2[rt][ct][1], ef[rt].x, pf[ct].y - pf[ct].x);
            dmma(k3[rt][ct][0], k3[rt][ct][1], ef[rt].y, pf[ct].x + pf[ct].y);
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
            S[((col >> 4) * CHI + rt * 8 + g) * MMA_S_STRIDE + (col & 15)] =
                cmake(k1[rt][ct][j] - k3[rt][ct][j], k1[rt][ct][j] + k2[rt][ct][j]);
          }
    }
    __syncwarp();   // E is dead and S is complete: prefetch the next parent
    if (k + 1 < count) stage_parent_padded(p, b, gidx + stride, E, lane);
    cp_async_commit();
    for (int cls = 0; cls < 2; ++cls) {
      if (!(grp.classes & (1 << cls))) continue;
      // Every trie environment is Hermitian (E' = sum_ij P_ij A_i^H E A_j with P
      // and the root Hermitian), so the children are too: only the tiles (0,0),
      // (0,1) and (1,1) are formed, the (1,0) tile is the conjugate transpose of
      // (0,1). I/Z: t0 = A_0^H S_0 and t1 = A_1^H S_1. X/Y: t0 = A_0^H S_1 (all
      // four tiles) and t1 = A_1^H S_0 = t0^H, transposed through the S panel.
      double ar[2][2][2], ai[2][2][2], br[2][2][2], bi[2][2][2];
      if (cls == 0) {
        class_tiles<GAUSS, true>(A, 0, S, 0, ar, ai, g, t);
        class_tiles<GAUSS, true>(A, CHI, S, 1, br, bi, g, t);
      } else {
        class_tiles<GAUSS, false>(A, 0, S, 1, ar, ai, g, t);
        __syncwarp();   // the panel is consumed: t0 goes into its place
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
        if (node.env_slot >= 0) {
          cplx *dst = p.env_cur + ((size_t)b * p.nslot_cur + node.env_slot) * ENV_ELEMS;
#pragma unroll
          for (int rt = 0; rt < 2; ++rt)
#pragma unroll
            for (int ct = rt; ct < 2; ++ct)
#pragma unroll
              for (int j = 0; j < 2; ++j) dst[(rt * 8 + g) * CHI + ct * 8 + 2 * t + j] = out[rt][ct][j];
#pragma unroll
          for (int j = 0; j < 2; ++j) dst[(8 + 2 * t + j) * CHI + g] = cconj(out[0][1][j]);
        }
        if (node.leaf >= 0) {
          double v = 0.0;
#pragma unroll
          for (int rt = 0; rt < 2; ++rt)
#pragma unroll
            for (int ct = rt; ct < 2; ++ct)
#pragma unroll
              for (int j = 0; j < 2; ++j) {
                const cplx rv = R[(rt * 8 + g) * CHI + ct * 8 + 2 * t + j];
                v += out[rt][ct][j].x * rv.x - out[rt][ct][j].y * rv.y;
              }
#pragma unroll
          for (int j = 0; j < 2; ++j) {   // the (1,0) tile: Re(conj(o) r)
            const cplx rv = R[(8 + 2 * t + j) * CHI + g];
            v += out[0][1][j].x * rv.x + out[0][1][j].y * rv.y;
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

__global__ void __launch_bounds__(MPF_WARPS * 32, 3)
level_mma_pf_kernel(LevelParams p, int groups_per_warp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  level_mma_pf_body<false>(p, groups_per_warp, smem_raw);
}

// The same level with Gauss's three-product complex multiply (a quarter fewer
// DMMA issues per product).
__global__ void __launch_bounds__(MPF_WARPS * 32, 3)
level_mma3_pf_kernel(LevelParams p, int groups_per_warp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  level_mma_pf_body<true>(p, groups_per_warp, smem_raw);
}

}  // namespace vqemps
