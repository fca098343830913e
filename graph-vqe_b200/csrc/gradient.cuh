// Adjoint (reverse-mode) gradient of the energy through the exact bond-doubling MPS.
//
// Reference: test/tools/reverse_mps.py:39-99 (ReverseMPS.sites / energy_chunk /
// value_gradient), which obtains the same quantity from torch autograd.
//
// B200 design.
// * Forward state. A CX on sites (s, s+1) doubles their shared bond without an
//   SVD: the left site becomes A (x) I on its right index and the right site
//   stack(B, flip B) on its left index (reverse_mps.py:45-50). Each site's tensor
//   therefore evolves independently of its neighbours, so a CTA per
//   (state, site) replays that site's own event list (one-site gates and its
//   half of each CX).
// * Energy. The same shared-prefix trie as the analytic path. The forward sweep
//   keeps the environments of every K-th level only (checkpoints; K = 1 keeps
//   all) and each CTA sums c_leaf * E_leaf of its leaves per level. The
//   backward sweep walks segments of K levels from the last: it recomputes the
//   segment's K - 1 inner levels from the checkpoint before it, then runs the
//   segment's backward levels.
// * Backward through the trie. For a parent E with children x and cotangents
//   Ebar_x (Re<Ebar, dE> convention): D_00 = Ebar_I + Ebar_Z, D_11 = Ebar_I - Ebar_Z,
//   D_01 = Ebar_X + i Ebar_Y, D_10 = Ebar_X - i Ebar_Y;
//   Ebar_parent = sum_{ii'} A_i D_ii' A_i'^H and
//   Abar_i += 2 sum_i' (E A_i') C_ii' with C_00 = D_00, C_11 = D_11, C_01 = D_10,
//   C_10 = D_01. A leaf closed against the identity right environment R_{s+1}
//   contributes c conj(R_{s+1}) to its cotangent; the right environments'
//   own cotangent is folded into one left sweep F_{q+1} = sum_i A_i^H F_q A_i +
//   (sum of c E_leaf at level q) giving Abar_q,i += 2 F_q A_q,i conj(R_{q+1}).
// * Backward through the circuit: per (state, site), the events are undone in
//   reverse (rotations are unitary, doublings are index maps), so no tape is
//   stored; dE/dtheta += Re<Abar, m'(theta) A_before> per rotation.
// Every reduction runs in a fixed order: the result is bitwise reproducible.
#pragma once
#include "common.cuh"
#include "evolve.cuh"
#include "expect.cuh"

namespace vqemps {

enum : int32_t { GOP_ONE = 0, GOP_CX = 1 };
enum : int32_t { EV_ONE = 0, EV_CXL = 1, EV_CXR = 2 };

struct GradOp {        // circuit-order op of the bond-doubling path
  int32_t kind;        // GOP_ONE / GOP_CX
  int32_t site;        // target site (ONE) or left site of the pair (CX)
  int32_t mat;         // fixed matrix offset or -1
  int32_t rot;         // ROT_* when mat < 0
  int32_t param;       // ONE: parameter or -1; CX: 0 if the control is the left site, else 1
  int32_t pad;
  double angle;
};

struct SiteEvent {     // one event in a single site's history
  int32_t kind;        // EV_ONE / EV_CXL (site is the left one) / EV_CXR
  int32_t ctrl_left;   // CX: control on the left site
  int32_t mat;
  int32_t rot;
  int32_t param;
  int32_t slot;        // gradient slot of a parametrised rotation, else -1
  double angle;
};

constexpr int GSITE_THREADS = 128;

__device__ __forceinline__ void event_matrix(const SiteEvent &e, const cplx *mats,
                                             const double *theta_b, cplx m[4], cplx dm[4]) {
  if (e.mat >= 0) {
    for (int i = 0; i < 4; ++i) { m[i] = mats[e.mat + i]; dm[i] = cmake(0, 0); }
    return;
  }
  const double ang = e.param >= 0 ? theta_b[e.param] * e.angle : e.angle;
  double s, c;
  sincos(0.5 * ang, &s, &c);
  const double hs = 0.5 * s, hc = 0.5 * c;
  if (e.rot == ROT_Y) {
    m[0] = cmake(c, 0); m[1] = cmake(-s, 0); m[2] = cmake(s, 0); m[3] = cmake(c, 0);
    dm[0] = cmake(-hs, 0); dm[1] = cmake(-hc, 0); dm[2] = cmake(hc, 0); dm[3] = cmake(-hs, 0);
  } else if (e.rot == ROT_X) {
    m[0] = cmake(c, 0); m[1] = cmake(0, -s); m[2] = cmake(0, -s); m[3] = cmake(c, 0);
    dm[0] = cmake(-hs, 0); dm[1] = cmake(0, -hc); dm[2] = cmake(0, -hc); dm[3] = cmake(-hs, 0);
  } else {
    m[0] = cmake(c, -s); m[1] = cmake(0, 0); m[2] = cmake(0, 0); m[3] = cmake(c, s);
    // d/dt exp(-+ i t/2) = -+ i/2 exp(-+ i t/2)
    dm[0] = cmake(-hs, -hc); dm[1] = cmake(0, 0); dm[2] = cmake(0, 0); dm[3] = cmake(-hs, hc);
  }
}

// ---------------------------------------------------------------------------
// forward: bond-doubling site tensors, CTA per (site, state)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(GSITE_THREADS)
grad_sites_kernel(const SiteEvent *__restrict__ events, const int32_t *__restrict__ ev_off,
                  const cplx *__restrict__ mats, const double *__restrict__ theta, int P, int n,
                  cplx init0, cplx init1, cplx *__restrict__ sites) {
  __shared__ cplx T0[SITE_ELEMS], T1[SITE_ELEMS];
  __shared__ cplx M[4];
  const int q = blockIdx.x, b = blockIdx.y, tid = threadIdx.x;
  const double *theta_b = theta + (size_t)b * P;
  for (int e = tid; e < SITE_ELEMS; e += GSITE_THREADS)
    T0[e] = e == 0 ? init0 : (e == CHI ? init1 : cmake(0, 0));
  int dl = 1, dr = 1;
  cplx *cur = T0, *nxt = T1;
  __syncthreads();
  for (int k = ev_off[q]; k < ev_off[q + 1]; ++k) {
    const SiteEvent ev = events[k];
    if (ev.kind == EV_ONE) {
      if (tid == 0) {
        cplx dm[4];
        event_matrix(ev, mats, theta_b, M, dm);
      }
      __syncthreads();
      for (int e = tid; e < CHI * CHI; e += GSITE_THREADS) {
        const int l = e >> 4, r = e & 15;
        const cplx a0 = cur[(l * 2 + 0) * CHI + r], a1 = cur[(l * 2 + 1) * CHI + r];
        cur[(l * 2 + 0) * CHI + r] = cadd(cmul(M[0], a0), cmul(M[1], a1));
        cur[(l * 2 + 1) * CHI + r] = cadd(cmul(M[2], a0), cmul(M[3], a1));
      }
    } else if (ev.kind == EV_CXL) {
      // new[a][i][b*2+s]: control left -> A[a][i][b] delta_{is}; target left -> A[a][i^s][b]
      for (int e = tid; e < SITE_ELEMS; e += GSITE_THREADS) {
        const int a = e >> 5, i = (e >> 4) & 1, col = e & 15;
        const int bb = col >> 1, s = col & 1;
        cplx v = cmake(0, 0);
        if (bb < dr) {
          if (ev.ctrl_left) v = (i == s) ? cur[(a * 2 + i) * CHI + bb] : cmake(0, 0);
          else v = cur[(a * 2 + (i ^ s)) * CHI + bb];
        }
        nxt[e] = v;
      }
      dr *= 2;
      cplx *t = cur; cur = nxt; nxt = t;
    } else {
      // new[b*2+s][j][r]: control left (site is target) -> B[b][j^s][r];
      //                   control right (site is control) -> B[b][j][r] delta_{js}
      for (int e = tid; e < SITE_ELEMS; e += GSITE_THREADS) {
        const int row = e >> 5, j = (e >> 4) & 1, r = e & 15;
        const int bb = row >> 1, s = row & 1;
        cplx v = cmake(0, 0);
        if (bb < dl) {
          if (ev.ctrl_left) v = cur[(bb * 2 + (j ^ s)) * CHI + r];
          else v = (j == s) ? cur[(bb * 2 + j) * CHI + r] : cmake(0, 0);
        }
        nxt[e] = v;
      }
      dl *= 2;
      cplx *t = cur; cur = nxt; nxt = t;
    }
    __syncthreads();
  }
  cplx *dst = sites + ((size_t)b * n + q) * SITE_ELEMS;
  for (int e = tid; e < SITE_ELEMS; e += GSITE_THREADS) dst[e] = cur[e];
}

// ---------------------------------------------------------------------------
// forward trie level keeping every environment; per-CTA sums of c * E_leaf
// ---------------------------------------------------------------------------
constexpr int GLEVEL_WARPS = 4;
constexpr int GROUPS_PER_WARP = 4;

struct GradLevelParams {
  const cplx *sites;
  const cplx *right;
  const cplx *env_prev;     // environments of level s-1 for state 0 (unused at s = 0)
  size_t prev_stride;       // elements between consecutive states
  cplx *env_cur;            // where level s environments go (state 0)
  size_t cur_stride;
  int leaf_work;            // forward: 1 computes leaf values and leaf sums, 0 only environments
  const DevGroup *groups;
  const DevNode *nodes;
  const double *leaf_coef;
  double *leafval;          // B x nleaf
  int nleaf;
  cplx *partial;            // B x gridDim.x x ENV_ELEMS (leaf sums) or B x gridDim.x x SITE_ELEMS (abar)
  cplx *bar_prev;           // backward: cotangents of level s-1 slots (B x maxslot)
  const cplx *bar_cur;      // backward: cotangents of level s slots
  int maxslot;
  int ngroups, n, s;
  // Suffix levels of the split evaluation (DMMA kernels only): sites holds the
  // transposed site tensors, a group without a parent slot starts from the
  // identity right environment R_{s+1}, and the backward writes that group's
  // parent cotangent (the cotangent of R_{s+1}) to rootbar[b][s].
  int suffix;
  cplx *rootbar;            // B x n x ENV_ELEMS
  // Real-gate kernels (grad_*_level_real_a_kernel): an environment of one kind
  // is stored as its nonzero part only, ENV_ELEMS doubles at the start of its
  // slot, unless env_complex is set for the level written -- the split plan's
  // cut levels, which the pair kernels read.
  int env_complex;
};

struct GradFwdSmem {
  cplx A[SITE_ELEMS];
  cplx E[GLEVEL_WARPS][ENV_ELEMS];
  cplx S[GLEVEL_WARPS][2 * ENV_ELEMS];
  cplx L[GLEVEL_WARPS][ENV_ELEMS];   // per-warp leaf sums
};

// S_i = E A_i for the 16 x 32 panel [S_0 | S_1]; lane tile 4 x 4.
__device__ __forceinline__ void panel_EA(const cplx *E, const cplx *A, cplx *S, int lane) {
  const int rt = lane >> 3, ct = lane & 7;
  cplx acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = cmake(0, 0);
#pragma unroll 4
  for (int k = 0; k < CHI; ++k) {
    cplx e[4], a[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) e[r] = E[(rt * 4 + r) * CHI + k];
#pragma unroll
    for (int c = 0; c < 4; ++c) a[c] = A[k * 2 * CHI + ct * 4 + c];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) cfma(acc[r][c], e[r], a[c]);
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int col = ct * 4 + c;
      S[(col >> 4) * ENV_ELEMS + (rt * 4 + r) * CHI + (col & 15)] = acc[r][c];
    }
}

__global__ void __launch_bounds__(GLEVEL_WARPS * 32)
grad_fwd_level_kernel(GradLevelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GradFwdSmem &sm = *reinterpret_cast<GradFwdSmem *>(smem_raw);
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
  for (int e = threadIdx.x; e < SITE_ELEMS; e += GLEVEL_WARPS * 32) sm.A[e] = ag[e];
  cplx *E = sm.E[warp];
  cplx *S = sm.S[warp];
  cplx *L = sm.L[warp];
  for (int e = lane; e < ENV_ELEMS; e += 32) L[e] = cmake(0, 0);
  __syncthreads();
  const cplx *A = sm.A;
  const int per_cta = GLEVEL_WARPS * GROUPS_PER_WARP;
  const int g0 = blockIdx.x * per_cta;
  const int g1 = min(g0 + per_cta, p.ngroups);
  const int rb = lane >> 3, cb = lane & 7;
  const cplx *R = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
  for (int gidx = g0 + warp; gidx < g1; gidx += GLEVEL_WARPS) {
    const DevGroup grp = p.groups[gidx];
    if (grp.parent_slot < 0) {
      for (int e = lane; e < ENV_ELEMS; e += 32) E[e] = cmake(e == 0 ? 1.0 : 0.0, 0.0);
    } else {
      const cplx *src = p.env_prev + (size_t)b * p.prev_stride + (size_t)grp.parent_slot * ENV_ELEMS;
      for (int e = lane; e < ENV_ELEMS; e += 32) E[e] = src[e];
    }
    __syncwarp();
    panel_EA(E, A, S, lane);
    __syncwarp();
    for (int cls = 0; cls < 2; ++cls) {
      if (!(grp.classes & (1 << cls))) continue;
      cplx t0[4][2], t1[4][2];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c) { t0[r][c] = cmake(0, 0); t1[r][c] = cmake(0, 0); }
      const int s0 = cls == 0 ? 0 : 1, s1 = cls == 0 ? 1 : 0;
#pragma unroll 2
      for (int a = 0; a < CHI; ++a) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const cplx av0 = A[(a * 2 + 0) * CHI + rb * 4 + r];
          const cplx av1 = A[(a * 2 + 1) * CHI + rb * 4 + r];
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            cfma_conj(t0[r][c], av0, S[s0 * ENV_ELEMS + a * CHI + cb * 2 + c]);
            cfma_conj(t1[r][c], av1, S[s1 * ENV_ELEMS + a * CHI + cb * 2 + c]);
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
          cplx *dst = p.env_cur + (size_t)b * p.cur_stride + (size_t)node.env_slot * ENV_ELEMS;
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 2; ++c) dst[(rb * 4 + r) * CHI + cb * 2 + c] = out[r][c];
        }
        if (node.leaf >= 0 && p.leaf_work) {
          const double cf = p.leaf_coef[node.leaf];
          double v = 0.0;
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
              const int idx = (rb * 4 + r) * CHI + cb * 2 + c;
              const cplx rv = R[idx];
              v += out[r][c].x * rv.x - out[r][c].y * rv.y;
              L[idx] = cadd(L[idx], cscale(out[r][c], cf));
            }
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) p.leafval[(size_t)b * p.nleaf + node.leaf] = v;
        }
      }
    }
    __syncwarp();
  }
  __syncthreads();
  if (!p.leaf_work) return;
  // fixed-order combination of the warps' leaf sums
  cplx *dst = p.partial + ((size_t)b * gridDim.x + blockIdx.x) * ENV_ELEMS;
  for (int e = threadIdx.x; e < ENV_ELEMS; e += GLEVEL_WARPS * 32) {
    cplx acc = sm.L[0][e];
    for (int w = 1; w < GLEVEL_WARPS; ++w) acc = cadd(acc, sm.L[w][e]);
    dst[e] = acc;
  }
}

// out[b][elem] (+)= sum over parts of partial[b][part][elem], fixed order.
__global__ void partial_sum_kernel(const cplx *__restrict__ partial, int parts, int elems,
                                   cplx *__restrict__ out, size_t out_stride, int accumulate) {
  const int b = blockIdx.y;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= elems) return;
  cplx acc = accumulate ? out[(size_t)b * out_stride + e] : cmake(0, 0);
  const cplx *src = partial + (size_t)b * parts * elems + e;
  for (int k = 0; k < parts; ++k) acc = cadd(acc, src[(size_t)k * elems]);
  out[(size_t)b * out_stride + e] = acc;
}

// out[b][a][i][c] += sum over parts of partial[b][part][c][i][a], fixed order:
// site cotangents of the split evaluation's suffix levels (transposed sites).
__global__ void partial_sum_t_kernel(const cplx *__restrict__ partial, int parts, cplx *__restrict__ out,
                                     size_t out_stride) {
  const int b = blockIdx.y;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= SITE_ELEMS) return;
  const int a = e >> 5, i = (e >> 4) & 1, c = e & 15;
  const cplx *src = partial + (size_t)b * parts * SITE_ELEMS + c * 32 + i * 16 + a;
  cplx acc = out[(size_t)b * out_stride + e];
  for (int k = 0; k < parts; ++k) acc = cadd(acc, src[(size_t)k * SITE_ELEMS]);
  out[(size_t)b * out_stride + e] = acc;
}

// Cotangents of the split evaluation's pair closures <P> = Re sum L o R with
// weight c (the pair's leaf coefficient): Lbar[j] = sum_p c_p conj(R[rs_p]) over
// the pairs of prefix slot j, Rbar[r] = sum_p c_p conj(L[ls_p]) over those of
// suffix slot r, each in pair order. Block (slot, state), thread per element.
// sign (may be null): Re(i^(kL + kR)) per pair; pairs where it is zero are left
// out -- for real states their value is zero at every angle (the cotangents of
// the real-gate gradient, whose imaginary-part bits they would only touch).
__global__ void __launch_bounds__(ENV_ELEMS)
split_pair_bwd_kernel(const cplx *__restrict__ left, size_t left_stride, const cplx *__restrict__ right,
                      size_t right_stride, const int32_t *__restrict__ pairs, const double *__restrict__ coef,
                      const int32_t *__restrict__ pl_off, int nls, const int32_t *__restrict__ pr_off,
                      const int32_t *__restrict__ pr_idx, cplx *__restrict__ lbar, size_t lbar_stride,
                      cplx *__restrict__ rbar, size_t rbar_stride, const double *__restrict__ sign) {
  const int b = blockIdx.y, e = threadIdx.x;
  const int j = blockIdx.x;
  cplx acc = cmake(0, 0);
  if (j < nls) {
    for (int k = pl_off[j]; k < pl_off[j + 1]; ++k) {
      if (sign && sign[k] == 0.0) continue;
      const cplx r = right[(size_t)b * right_stride + (size_t)pairs[3 * k + 1] * ENV_ELEMS + e];
      acc = cadd(acc, cscale(cconj(r), coef[pairs[3 * k + 2]]));
    }
    lbar[(size_t)b * lbar_stride + (size_t)j * ENV_ELEMS + e] = acc;
  } else {
    const int r = j - nls;
    for (int q = pr_off[r]; q < pr_off[r + 1]; ++q) {
      const int k = pr_idx[q];
      if (sign && sign[k] == 0.0) continue;
      const cplx l = left[(size_t)b * left_stride + (size_t)pairs[3 * k] * ENV_ELEMS + e];
      acc = cadd(acc, cscale(cconj(l), coef[pairs[3 * k + 2]]));
    }
    rbar[(size_t)b * rbar_stride + (size_t)r * ENV_ELEMS + e] = acc;
  }
}

// ---------------------------------------------------------------------------
// suffix part: F_0 = c_identity e00; Abar_q,i = 2 F_q A_q,i conj(R_{q+1});
// F_{q+1} = sum_i A_i^H F_q A_i + leafsum[q].  One CTA per state.
// ---------------------------------------------------------------------------
// rootbar (may be null): cotangents of R_{q+1} from the split evaluation's
// suffix roots (bar convention, conjugated into F); accumulate adds the site
// cotangents to sitebar instead of writing them.  The sweep covers sites
// q0 .. q1-1: it starts from fstate[b] when q0 > 0 and stores F_{q1} there when
// q1 < n, so a sweep split at the cut gives the same bits as one sweep.
__global__ void __launch_bounds__(256)
grad_suffix_kernel(const cplx *__restrict__ sites, const cplx *__restrict__ right,
                   const cplx *__restrict__ leafsum, const cplx *__restrict__ rootbar,
                   double identity_coef, int n, int accumulate, cplx *__restrict__ sitebar, int q0, int q1,
                   cplx *__restrict__ fstate) {
  __shared__ cplx A[SITE_ELEMS];
  __shared__ cplx F[ENV_ELEMS];
  __shared__ cplx Rc[ENV_ELEMS];
  __shared__ cplx Tm[SITE_ELEMS];
  const int b = blockIdx.x, tid = threadIdx.x;
  F[tid] = q0 > 0 ? fstate[(size_t)b * ENV_ELEMS + tid] : cmake(tid == 0 ? identity_coef : 0.0, 0.0);
  for (int q = q0; q < q1; ++q) {
    const cplx *ag = sites + ((size_t)b * n + q) * SITE_ELEMS;
    A[tid] = ag[tid];
    A[tid + 256] = ag[tid + 256];
    Rc[tid] = cconj(right[((size_t)b * (n + 1) + q + 1) * ENV_ELEMS + tid]);
    __syncthreads();
    // Tm[a][i][c] = sum_a' F[a][a'] A[a'][i][c]
    for (int e = tid; e < SITE_ELEMS; e += 256) {
      const int a = e >> 5, ic = e & 31;
      cplx acc = cmake(0, 0);
      for (int ap = 0; ap < CHI; ++ap) cfma(acc, F[a * CHI + ap], A[ap * 2 * CHI + ic]);
      Tm[e] = acc;
    }
    __syncthreads();
    // Abar[a][i][c] = 2 sum_c' Tm[a][i][c'] conj(R)[c'][c]
    cplx *dst = sitebar + ((size_t)b * n + q) * SITE_ELEMS;
    for (int e = tid; e < SITE_ELEMS; e += 256) {
      const int ai = e >> 4, c = e & 15;
      cplx acc = cmake(0, 0);
      for (int cp = 0; cp < CHI; ++cp) cfma(acc, Tm[ai * CHI + cp], Rc[cp * CHI + c]);
      dst[e] = accumulate ? cadd(dst[e], cscale(acc, 2.0)) : cscale(acc, 2.0);
    }
    // F' = sum_i A_i^H Tm_i + leafsum[q] (+ conj(rootbar[q]))
    {
      const int bb = tid >> 4, c = tid & 15;
      cplx acc = leafsum[((size_t)b * n + q) * ENV_ELEMS + tid];
      if (rootbar) acc = cadd(acc, cconj(rootbar[((size_t)b * n + q) * ENV_ELEMS + tid]));
      for (int a = 0; a < CHI; ++a) {
        cfma_conj(acc, A[(a * 2 + 0) * CHI + bb], Tm[(a * 2 + 0) * CHI + c]);
        cfma_conj(acc, A[(a * 2 + 1) * CHI + bb], Tm[(a * 2 + 1) * CHI + c]);
      }
      __syncthreads();
      F[tid] = acc;
    }
    __syncthreads();
  }
  if (q1 < n) fstate[(size_t)b * ENV_ELEMS + tid] = F[tid];
}

// ---------------------------------------------------------------------------
// backward trie level: parent cotangents and per-CTA site cotangent partials
// ---------------------------------------------------------------------------
struct GradBwdSmem {
  cplx A[SITE_ELEMS];
  cplx S[GLEVEL_WARPS][2 * ENV_ELEMS];    // E (first half) then S_0 | S_1, later Y_0 | Y_1
  cplx C[GLEVEL_WARPS][2 * ENV_ELEMS];    // a pair of C / D matrices
  cplx Ab[GLEVEL_WARPS][SITE_ELEMS];      // per-warp site cotangent accumulator
};

// acc[r][c] (4 x 4 lane tile over a 16 x 32 panel) += sum_k X_sel(k)[row][k] Y[k][col]
// Used twice: Abar panel += S_i' C_ii' and Y panel += A_i D_ii'.
__global__ void __launch_bounds__(GLEVEL_WARPS * 32)
grad_bwd_level_kernel(GradLevelParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  GradBwdSmem &sm = *reinterpret_cast<GradBwdSmem *>(smem_raw);
  const int b = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const cplx *ag = p.sites + ((size_t)b * p.n + p.s) * SITE_ELEMS;
  for (int e = threadIdx.x; e < SITE_ELEMS; e += GLEVEL_WARPS * 32) sm.A[e] = ag[e];
  cplx *S = sm.S[warp];
  cplx *C = sm.C[warp];
  cplx *Ab = sm.Ab[warp];
  for (int e = lane; e < SITE_ELEMS; e += 32) Ab[e] = cmake(0, 0);
  __syncthreads();
  const cplx *A = sm.A;
  const int per_cta = GLEVEL_WARPS * GROUPS_PER_WARP;
  const int g0 = blockIdx.x * per_cta;
  const int g1 = min(g0 + per_cta, p.ngroups);
  const cplx *R = p.right + ((size_t)b * (p.n + 1) + p.s + 1) * ENV_ELEMS;
  const int rt = lane >> 3, ct = lane & 7;
  for (int gidx = g0 + warp; gidx < g1; gidx += GLEVEL_WARPS) {
    const DevGroup grp = p.groups[gidx];
    // parent environment into C[0..255], then S = E [A_0 | A_1]
    if (grp.parent_slot < 0) {
      for (int e = lane; e < ENV_ELEMS; e += 32) C[e] = cmake(e == 0 ? 1.0 : 0.0, 0.0);
    } else {
      const cplx *src = p.env_prev + (size_t)b * p.prev_stride + (size_t)grp.parent_slot * ENV_ELEMS;
      for (int e = lane; e < ENV_ELEMS; e += 32) C[e] = src[e];
    }
    __syncwarp();
    panel_EA(C, A, S, lane);
    __syncwarp();
    // child cotangents
    int idx_child[4] = {-1, -1, -1, -1};
    for (int ci = 0; ci < grp.nchild; ++ci) idx_child[p.nodes[grp.child_begin + ci].code] = grp.child_begin + ci;
    // Y panel accumulators (Y_0 | Y_1), lane tile 4 x 4 over 16 x 32
    cplx ya[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) ya[r][c] = cmake(0, 0);
    for (int cls = 0; cls < 2; ++cls) {
      if (!(grp.classes & (1 << cls))) continue;
      // cls 0: C holds (D_00, D_11) = (Ebar_I + Ebar_Z, Ebar_I - Ebar_Z)
      // cls 1: C holds (D_01, D_10) = (Ebar_X + i Ebar_Y, Ebar_X - i Ebar_Y)
      const int ca = idx_child[cls == 0 ? 0 : 1], cbx = idx_child[cls == 0 ? 3 : 2];
      DevNode na{}, nb{};
      na.env_slot = nb.env_slot = -1; na.leaf = nb.leaf = -1;
      if (ca >= 0) na = p.nodes[ca];
      if (cbx >= 0) nb = p.nodes[cbx];
      const double cfa = na.leaf >= 0 ? p.leaf_coef[na.leaf] : 0.0;
      const double cfb = nb.leaf >= 0 ? p.leaf_coef[nb.leaf] : 0.0;
      const cplx *bara = na.env_slot >= 0 ? p.bar_cur + ((size_t)b * p.maxslot + na.env_slot) * ENV_ELEMS : nullptr;
      const cplx *barb = nb.env_slot >= 0 ? p.bar_cur + ((size_t)b * p.maxslot + nb.env_slot) * ENV_ELEMS : nullptr;
      for (int e = lane; e < ENV_ELEMS; e += 32) {
        const cplx rc = cconj(R[e]);
        cplx xa = cscale(rc, cfa), xb = cscale(rc, cfb);
        if (bara) xa = cadd(xa, bara[e]);
        if (barb) xb = cadd(xb, barb[e]);
        if (cls == 0) {
          C[e] = cadd(xa, xb);
          C[ENV_ELEMS + e] = csub(xa, xb);
        } else {
          const cplx ixb = cmake(-xb.y, xb.x);
          C[e] = cadd(xa, ixb);
          C[ENV_ELEMS + e] = csub(xa, ixb);
        }
      }
      __syncwarp();
      // Abar panel: cls 0: Abar_0 += 2 S_0 D_00, Abar_1 += 2 S_1 D_11
      //             cls 1: Abar_0 += 2 S_1 C_01 = 2 S_1 D_10, Abar_1 += 2 S_0 C_10 = 2 S_0 D_01
      // Y panel:    cls 0: Y_0 += A_0 D_00, Y_1 += A_1 D_11
      //             cls 1: Y_0 += A_1 D_10, Y_1 += A_0 D_01
      {
        cplx aa[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) aa[r][c] = cmake(0, 0);
        // panel column block i = ct >> 2 (0: Abar_0 / Y_0, 1: Abar_1 / Y_1)
        const int iout = ct >> 2;
        const int src_s = cls == 0 ? iout : 1 - iout;             // which S_i' multiplies
        const int dsel = cls == 0 ? iout : 1 - iout;              // D_00/D_11 or D_10/D_01 slot
        const int asel = cls == 0 ? iout : 1 - iout;              // which A_i for Y
        const cplx *Dm = C + dsel * ENV_ELEMS;
#pragma unroll 4
        for (int k = 0; k < CHI; ++k) {
          cplx sv[4], avv[4], dv[4];
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            sv[r] = S[src_s * ENV_ELEMS + (rt * 4 + r) * CHI + k];
            avv[r] = A[((rt * 4 + r) * 2 + asel) * CHI + k];
          }
#pragma unroll
          for (int c = 0; c < 4; ++c) dv[c] = Dm[k * CHI + (ct & 3) * 4 + c];
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              cfma(aa[r][c], sv[r], dv[c]);
              cfma(ya[r][c], avv[r], dv[c]);
            }
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const int idx = ((rt * 4 + r) * 2 + iout) * CHI + (ct & 3) * 4 + c;
            Ab[idx] = cadd(Ab[idx], cscale(aa[r][c], 2.0));
          }
      }
      __syncwarp();
    }
    if (p.s > 0) {
      // Y panel to S (S no longer needed), then Ebar_parent = Y_0 A_0^H + Y_1 A_1^H
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int iout = ct >> 2;
          S[iout * ENV_ELEMS + (rt * 4 + r) * CHI + (ct & 3) * 4 + c] = ya[r][c];
        }
      __syncwarp();
      const int rb = lane >> 3, cb = lane & 7;
      cplx o[4][2];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c) o[r][c] = cmake(0, 0);
      // Ebar[x][y] = sum_i sum_k Y_i[x][k] conj(A[y][i][k])
#pragma unroll 2
      for (int k = 0; k < CHI; ++k) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          cplx yv[4], av[2];
#pragma unroll
          for (int r = 0; r < 4; ++r) yv[r] = S[i * ENV_ELEMS + (rb * 4 + r) * CHI + k];
#pragma unroll
          for (int c = 0; c < 2; ++c) av[c] = cconj(A[((cb * 2 + c) * 2 + i) * CHI + k]);
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 2; ++c) cfma(o[r][c], yv[r], av[c]);
        }
      }
      cplx *dst = p.bar_prev + ((size_t)b * p.maxslot + grp.parent_slot) * ENV_ELEMS;
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 2; ++c) dst[(rb * 4 + r) * CHI + cb * 2 + c] = o[r][c];
    }
    __syncwarp();
  }
  __syncthreads();
  cplx *dst = p.partial + ((size_t)b * gridDim.x + blockIdx.x) * SITE_ELEMS;
  for (int e = threadIdx.x; e < SITE_ELEMS; e += GLEVEL_WARPS * 32) {
    cplx acc = sm.Ab[0][e];
    for (int w = 1; w < GLEVEL_WARPS; ++w) acc = cadd(acc, sm.Ab[w][e]);
    dst[e] = acc;
  }
}

// ---------------------------------------------------------------------------
// backward through each site's events; per-rotation gradient contributions
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(GSITE_THREADS)
grad_circuit_kernel(const SiteEvent *__restrict__ events, const int32_t *__restrict__ ev_off,
                    const int32_t *__restrict__ dims_after, const cplx *__restrict__ mats,
                    const double *__restrict__ theta, int P, int n, const cplx *__restrict__ sites,
                    const cplx *__restrict__ sitebar, double *__restrict__ slot_grad, int nslots) {
  __shared__ cplx A0[SITE_ELEMS], A1[SITE_ELEMS], G0[SITE_ELEMS], G1[SITE_ELEMS];
  __shared__ cplx M[4], DM[4];
  __shared__ double red[GSITE_THREADS / 32];
  const int q = blockIdx.x, b = blockIdx.y, tid = threadIdx.x;
  const double *theta_b = theta + (size_t)b * P;
  const cplx *src = sites + ((size_t)b * n + q) * SITE_ELEMS;
  const cplx *gsrc = sitebar + ((size_t)b * n + q) * SITE_ELEMS;
  for (int e = tid; e < SITE_ELEMS; e += GSITE_THREADS) { A0[e] = src[e]; G0[e] = gsrc[e]; }
  cplx *a = A0, *an = A1, *g = G0, *gn = G1;
  __syncthreads();
  for (int k = ev_off[q + 1] - 1; k >= ev_off[q]; --k) {
    const SiteEvent ev = events[k];
    // dims of this site after event k (2 ints per event)
    const int dl = dims_after[2 * k], dr = dims_after[2 * k + 1];
    if (ev.kind == EV_ONE) {
      if (tid == 0) event_matrix(ev, mats, theta_b, M, DM);
      __syncthreads();
      // A_old = m^H A ; grad += Re sum conj(Abar) (m' A_old) ; Abar_old = m^H Abar
      double part = 0.0;
      for (int e = tid; e < CHI * CHI; e += GSITE_THREADS) {
        const int l = e >> 4, r = e & 15;
        const cplx x0 = a[(l * 2 + 0) * CHI + r], x1 = a[(l * 2 + 1) * CHI + r];
        const cplx o0 = cadd(cmul(cconj(M[0]), x0), cmul(cconj(M[2]), x1));
        const cplx o1 = cadd(cmul(cconj(M[1]), x0), cmul(cconj(M[3]), x1));
        const cplx g0 = g[(l * 2 + 0) * CHI + r], g1 = g[(l * 2 + 1) * CHI + r];
        if (ev.slot >= 0) {
          const cplx d0 = cadd(cmul(DM[0], o0), cmul(DM[1], o1));
          const cplx d1 = cadd(cmul(DM[2], o0), cmul(DM[3], o1));
          part += g0.x * d0.x + g0.y * d0.y + g1.x * d1.x + g1.y * d1.y;
        }
        a[(l * 2 + 0) * CHI + r] = o0;
        a[(l * 2 + 1) * CHI + r] = o1;
        g[(l * 2 + 0) * CHI + r] = cadd(cmul(cconj(M[0]), g0), cmul(cconj(M[2]), g1));
        g[(l * 2 + 1) * CHI + r] = cadd(cmul(cconj(M[1]), g0), cmul(cconj(M[3]), g1));
      }
      if (ev.slot >= 0) {
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if ((tid & 31) == 0) red[tid >> 5] = part;
        __syncthreads();
        if (tid == 0) {
          double t = 0.0;
          for (int w = 0; w < GSITE_THREADS / 32; ++w) t += red[w];
          slot_grad[(size_t)b * nslots + ev.slot] = t * (ev.param >= 0 ? ev.angle : 0.0);
        }
      }
    } else if (ev.kind == EV_CXL) {
      // forward: new[a][i][bb*2+s] from old (dl, 2, dr/2)
      const int drold = dr >> 1;
      for (int e = tid; e < SITE_ELEMS; e += GSITE_THREADS) {
        const int aa = e >> 5, i = (e >> 4) & 1, bb = e & 15;
        cplx vo = cmake(0, 0), go = cmake(0, 0);
        if (bb < drold && aa < dl) {
          if (ev.ctrl_left) {
            vo = a[(aa * 2 + i) * CHI + bb * 2 + i];
            go = g[(aa * 2 + i) * CHI + bb * 2 + i];
          } else {
            vo = a[(aa * 2 + i) * CHI + bb * 2 + 0];
            go = cadd(g[(aa * 2 + i) * CHI + bb * 2 + 0], g[(aa * 2 + (i ^ 1)) * CHI + bb * 2 + 1]);
          }
        }
        an[e] = vo;
        gn[e] = go;
      }
      cplx *t = a; a = an; an = t;
      t = g; g = gn; gn = t;
    } else {
      const int dlold = dl >> 1;
      for (int e = tid; e < SITE_ELEMS; e += GSITE_THREADS) {
        const int bb = e >> 5, j = (e >> 4) & 1, r = e & 15;
        cplx vo = cmake(0, 0), go = cmake(0, 0);
        if (bb < dlold && r < dr) {
          if (ev.ctrl_left) {
            vo = a[((bb * 2 + 0) * 2 + j) * CHI + r];
            go = cadd(g[((bb * 2 + 0) * 2 + j) * CHI + r], g[((bb * 2 + 1) * 2 + (j ^ 1)) * CHI + r]);
          } else {
            vo = a[((bb * 2 + j) * 2 + j) * CHI + r];
            go = g[((bb * 2 + j) * 2 + j) * CHI + r];
          }
        }
        an[e] = vo;
        gn[e] = go;
      }
      cplx *t = a; a = an; an = t;
      t = g; g = gn; gn = t;
    }
    __syncthreads();
  }
}

// grad[b][p] = sum of slot_grad over the slots of parameter p (CSR), fixed order.
__global__ void grad_param_kernel(const double *__restrict__ slot_grad, int nslots,
                                  const int32_t *__restrict__ off, const int32_t *__restrict__ slots,
                                  int P, double *__restrict__ grad, const int32_t *__restrict__ status) {
  const int b = blockIdx.y;
  const int pi = blockIdx.x * blockDim.x + threadIdx.x;
  if (pi >= P) return;
  double acc = 0.0;
  for (int k = off[pi]; k < off[pi + 1]; ++k) acc += slot_grad[(size_t)b * nslots + slots[k]];
  grad[(size_t)b * P + pi] = status[b] == 0 ? acc : __longlong_as_double(0x7ff8000000000000LL);
}

inline void grad_set_attributes() {
  cudaFuncSetAttribute(grad_fwd_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(GradFwdSmem));
  cudaFuncSetAttribute(grad_bwd_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(GradBwdSmem));
}

}  // namespace vqemps
