// State preparation: apply a compiled gate list to B parameter sets at once.
//
// Reference algorithm (test/backend/source):
//   apply1q / k_apply1qInPlace ........ sharded_mps.cuh:16-26, 465-474
//   apply2q / k_buildM ................ sharded_mps.cuh:30-45, 477-516
//   singleGpuSvdFactors ............... dist_svd.cuh:233-283 (cuSOLVER Zgesvd)
//   selectDirectSvdRank ............... dist_svd.cuh:194-212 (zero-cutoff rank guard)
//   packDirectSvdFactors .............. dist_svd.cuh:214-231 (left = U, right = S*Vh)
//
// B200 design: one CTA per parameter set walks the whole gate list; nothing
// returns to the host between gates (the reference synchronises twice per
// gate). One-qubit gates are not applied when they arrive: they accumulate in a
// per-site 2x2 matrix in shared memory and are folded into the next two-site
// gate's 4x4 matrix (or applied at the end). Each two-site gate builds
// Theta = G (A (x) B) (2Dl x 2Dr, <= 32 x 32 complex) in shared memory and
// factors it with an FP64 one-sided Jacobi SVD on its shorter side. For a wide
// or square Theta the ROWS are orthogonalised by left unitary rotations,
// V^H Theta = X, so the new left site V[:, kept] is unitary to rounding (no
// division by small singular values, null directions included) and the right
// site is the kept rows of X = S * Vh. For a tall Theta (the left-to-right
// sweeps at full bond: 32 x 16) the same rotations act on Theta^T, halving the
// vectors and quartering the rotation steps; the left site is then the
// normalised rotated columns, re-orthogonalised against each other where a
// singular value is numerically zero. Singular values are kept in descending
// order, the gesvd ordering the reference uses.
//
// Which factor carries the singular values is a gauge choice: the state, the
// kept bond dimension, the rank guard and every observable are the same either
// way. The reference packs left = U, right = S V^H (dist_svd.cuh:214-231). The
// circuit compiler flags a gate GATE_SIGMA_LEFT (left = U S, right = V^H) when
// the next two-site gate that touches its sites touches only its right site:
// the next Theta then takes this gate's isometric factor, its rows start closer
// to orthogonal, and the Jacobi SVD needs far fewer sweeps (on the 40-qubit
// benchmark chain, whose sweeps run left to right, 5.6 instead of 9.6 sweeps
// per 16-row Theta, 4,069 instead of 7,177 Jacobi steps per state).
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"

namespace vqemps {

enum : int32_t { GATE_ONE = 0, GATE_TWO = 1 };
enum : int32_t { ROT_NONE = -1, ROT_X = 0, ROT_Y = 1, ROT_Z = 2 };

// GATE_TWO flags: the singular values go to the left factor (A_s = U S,
// A_{s+1} = V^H) instead of the right one (A_s = U, A_{s+1} = S V^H).
enum : int32_t { GATE_SIGMA_LEFT = 1 };

struct DevGate {
  int32_t kind;   // GATE_ONE / GATE_TWO
  int32_t site;   // target site (ONE) or left site s of the pair (s, s+1) (TWO)
  int32_t mat;    // offset of a fixed matrix in the matrix table, or -1 (rotation)
  int32_t rot;    // ROT_* when mat < 0
  int32_t param;  // parameter index or -1
  int32_t flags;  // GATE_SIGMA_LEFT (TWO)
  double angle;   // constant angle (param < 0) or scale (param >= 0)
};

struct EvolveParams {
  const DevGate *gates;
  int ngates;
  const cplx *mats;
  int n;
  int P;
  const double *theta;   // B x P
  cplx *sites;           // B x n x SITE_ELEMS
  int32_t *bonds;        // B x (n + 1)
  int32_t *status;       // B
  cplx init0, init1;     // initial single-qubit state
  int max_bond;
  double abs_cut, rel_cut;
  // Partition sets (st_part null for a uniform batch): state b belongs to
  // partition st_part[b] of width part_n[] and gates part_gate_off[k] ..
  // part_gate_off[k + 1]; n above is then the widest partition (the stride of
  // sites and bonds) and P the stride of theta rows.
  const int32_t *st_part;
  const int32_t *part_n;
  const int32_t *part_gate_off;
  // Two-CTA schedule (evolve_pair_kernel): step t applies gates sched[2t] and
  // sched[2t + 1] (-1: none) on disjoint site pairs; gate_q[4g .. 4g + 3] bounds
  // the pending one-site gates (qlist) folded into two-site gate g on its left
  // and right site; tail_off[x .. x + 1] the one-site gates after the last
  // two-site gate on site x. Partition sets: steps step_off[k] .. step_off[k + 1]
  // and tail entries from part_tail_off[k].
  const int32_t *sched;
  int nsteps;
  const int32_t *step_off;
  const int32_t *gate_q;
  const int32_t *qlist;
  const int32_t *tail_off;
  const int32_t *part_tail_off;
  // Mixed partition sets (the per-partition chain kernels): 1 where partition
  // k's circuit is of real gates (real-arithmetic Jacobi), 0 where complex.
  const int32_t *part_real;
  // Multi-CTA chains of one circuit: the pending one-site products of every
  // two-site gate, [B][ngates][8] (U_s then U_{s+1}), formed beforehand by
  // pending_kernel (null: formed by one thread when the gate is applied).
  const cplx *upend;
};

constexpr int EVOLVE_THREADS = 256;   // one-CTA gate chain
constexpr int PAIR_THREADS = 128;     // each CTA of the two-CTA gate chain
constexpr int JACOBI_MAX_SWEEPS = 40;

// Dynamic shared memory layout (bytes).
struct EvolveSmem {
  static constexpr int X = 0;                              // 32 x 32 cplx, [row][col]
  static constexpr int VT = X + 32 * 32 * 16;              // 32 x 32 cplx, [col][row] of V
  static constexpr int SA = VT + 32 * 32 * 16;             // site s tile
  static constexpr int SB = SA + SITE_ELEMS * 16;          // site s+1 tile
  static constexpr int G = SB + SITE_ELEMS * 16;           // fused 4x4
  static constexpr int NORM = G + 16 * 16;                 // 32 doubles
  static constexpr int SIG = NORM + 32 * 8;                // 32 sorted singular values
  static constexpr int PERM = SIG + 32 * 8;                // 32 ints
  static constexpr int MISC = PERM + 32 * 4;               // scalars
  static constexpr int SCHED = MISC + 64;                  // 32 x 16 ints: Jacobi pairs of the gate
  static constexpr int PEND = SCHED + 32 * 16 * 4;         // n x 4 cplx pending 1q matrices
  static __host__ __device__ int bytes(int n) { return PEND + n * 4 * 16 + (n + 1) * 4 + 16; }
};

// The same tiles for real arithmetic in the multi-CTA chains (two_site_update_real
// uses X, VT as 32 x 32 doubles, SA, SB as site tiles of doubles, G as 16
// doubles) plus the 8 pending one-site entries U_s, U_{s+1}: 26.9 KiB.
struct EvolveSmemReal {
  static constexpr int X = 0;                              // 32 x 32 doubles
  static constexpr int VT = X + 32 * 32 * 8;
  static constexpr int SA = VT + 32 * 32 * 8;              // site s tile, doubles
  static constexpr int SB = SA + SITE_ELEMS * 8;
  static constexpr int G = SB + SITE_ELEMS * 8;            // 4 x 4 doubles
  static constexpr int NORM = G + 16 * 8;
  static constexpr int SIG = NORM + 32 * 8;
  static constexpr int PERM = SIG + 32 * 8;
  static constexpr int MISC = PERM + 32 * 4;
  static constexpr int SCHED = MISC + 64;
  static constexpr int PEND = SCHED + 32 * 16 * 4;         // 8 cplx
  static __host__ __device__ int bytes(int) { return PEND + 8 * 16; }
};

__device__ __forceinline__ void one_site_matrix(const DevGate &g, const cplx *mats,
                                                const double *theta_b, cplx m[4]) {
  if (g.mat >= 0) {
    for (int i = 0; i < 4; ++i) m[i] = mats[g.mat + i];
    return;
  }
  double ang = g.param >= 0 ? theta_b[g.param] * g.angle : g.angle;
  double s, c;
  sincos(0.5 * ang, &s, &c);
  if (g.rot == ROT_Y) {
    m[0] = cmake(c, 0); m[1] = cmake(-s, 0); m[2] = cmake(s, 0); m[3] = cmake(c, 0);
  } else if (g.rot == ROT_X) {
    m[0] = cmake(c, 0); m[1] = cmake(0, -s); m[2] = cmake(0, -s); m[3] = cmake(c, 0);
  } else {
    m[0] = cmake(c, -s); m[1] = cmake(0, 0); m[2] = cmake(0, 0); m[3] = cmake(c, s);
  }
}

// u <- m u for 2 x 2 matrices (a one-site gate joining the pending product).
// Not inlined, so that both gate chains round it identically.
__device__ __noinline__ void left_multiply_2x2(const cplx *m, cplx *u) {
  const cplx u0 = u[0], u1 = u[1], u2 = u[2], u3 = u[3];
  u[0] = cadd(cmul(m[0], u0), cmul(m[1], u2));
  u[1] = cadd(cmul(m[0], u1), cmul(m[1], u3));
  u[2] = cadd(cmul(m[2], u0), cmul(m[3], u2));
  u[3] = cadd(cmul(m[2], u1), cmul(m[3], u3));
}

// a[l, i, r] <- sum_j u[i][j] a[l, j, r] for the entries e = tid, tid + step, ...
// of one site (a one-site matrix applied in place). Not inlined, as above.
__device__ __noinline__ void apply_2x2_to_site(const cplx *u, cplx *a, int tid, int step) {
  for (int e = tid; e < CHI * CHI; e += step) {
    const int l = e >> 4, r = e & 15;
    const cplx a0 = __ldcg(a + (l * 2 + 0) * CHI + r), a1 = __ldcg(a + (l * 2 + 1) * CHI + r);
    a[(l * 2 + 0) * CHI + r] = cadd(cmul(u[0], a0), cmul(u[1], a1));
    a[(l * 2 + 1) * CHI + r] = cadd(cmul(u[2], a0), cmul(u[3], a1));
  }
}

// One two-site gate on sites (s, s + 1) of one state, by the whole CTA: Theta =
// G (U_s (x) U_{s+1}) (A_s A_{s+1}), FP64 one-sided Jacobi SVD, rank selection and
// the packed factors written back to sites_b. us / ut: the pending one-site
// matrices of the two sites (reset to the identity here); gm: the 4 x 4 gate.
// Writes the new bond dimension to *bond_next; returns the status (uniform over
// the CTA; MISC[0] holds it too).
struct EvolveShared {
  cplx *X, *VT, *SA, *SB, *G;
  double *NORM, *SIG;
  int *PERM, *MISC, *SCHED;
};

// NORM[row] = sum_j |X[row][j]|^2 for rows < mr (even), 16 lanes per row, by
// the whole CTA of NT threads (the two 16-lane groups of a warp take rows
// 2w + (NT/16) t and 2w + 1 + (NT/16) t, so the width-16 shuffles run on uniform
// warps). The sum of a row does not depend on NT.
template <int NT>
__device__ __forceinline__ void jacobi_row_norms(const cplx *X, double *NORM, int mr, int mc, int tid) {
  const int grp = tid >> 4, lane = tid & 15;
  for (int row = grp; row < mr; row += NT / 16) {
    double a = 0.0;
    for (int j = lane; j < mc; j += 16) a += cabs2(X[row * 32 + j]);
    for (int o = 8; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o, 16);
    if (lane == 0) NORM[row] = a;
  }
}

template <int NT>
__device__ __forceinline__ int two_site_update(const EvolveParams &p, const EvolveShared &sh, cplx *sites_b, int s,
                                            int dl, int dc, int dr, cplx *us, cplx *ut, const cplx *gm,
                                            int *bond_next, bool sigma_left) {
  cplx *X = sh.X, *VT = sh.VT, *SA = sh.SA, *SB = sh.SB, *G = sh.G;
  double *NORM = sh.NORM, *SIG = sh.SIG;
  int *PERM = sh.PERM, *MISC = sh.MISC, *SCHED = sh.SCHED;
  const int tid = threadIdx.x;
  const double eps = 2.2204460492503131e-16;
    // ---- two-site gate on (s, s+1) ----
    const int m = 2 * dl, ncol = 2 * dr;
    // Jacobi runs on the shorter side: the rows of Theta when m <= ncol, the
    // rows of Theta^T (the columns of Theta) when Theta is tall.
    const bool tall = m > ncol;
    const int mr = tall ? ncol : m, mc = tall ? m : ncol;
    {
      const cplx *ga = sites_b + (size_t)s * SITE_ELEMS;
      const cplx *gb = ga + SITE_ELEMS;
      for (int e = tid; e < SITE_ELEMS; e += NT) { SA[e] = __ldcg(ga + e); SB[e] = __ldcg(gb + e); }
      if (tid < 16) {
        // G' = G (U_s (x) U_{s+1}); G'[IJ, ij] = sum_{i'j'} G[IJ, i'j'] U_s[i', i] U_{s+1}[j', j]
        const int row = tid >> 2, col = tid & 3;
        const int i = col >> 1, j = col & 1;
        cplx acc = cmake(0, 0);
        for (int ip = 0; ip < 2; ++ip)
          for (int jp = 0; jp < 2; ++jp)
            acc = cadd(acc, cmul(gm[row * 4 + ip * 2 + jp], cmul(us[ip * 2 + i], ut[jp * 2 + j])));
        G[tid] = acc;
      }
    }
    __syncthreads();
    if (tid < 4) {
      us[tid] = cmake(tid == 0 || tid == 3 ? 1 : 0, 0);
      ut[tid] = cmake(tid == 0 || tid == 3 ? 1 : 0, 0);
    }
    // Theta[(l*2+I), (J*dr+r)] = sum_ij G'[(I*2+J)*4+(i*2+j)] sum_c A[l,i,c] B[c,j,r]  (k_buildM)
    for (int lr = tid; lr < dl * dr; lr += NT) {
      const int l = lr / dr, r = lr % dr;
      cplx t00 = cmake(0, 0), t01 = cmake(0, 0), t10 = cmake(0, 0), t11 = cmake(0, 0);
      for (int c = 0; c < dc; ++c) {
        cplx a0 = SA[(l * 2 + 0) * CHI + c], a1 = SA[(l * 2 + 1) * CHI + c];
        cplx b0 = SB[(c * 2 + 0) * CHI + r], b1 = SB[(c * 2 + 1) * CHI + r];
        cfma(t00, a0, b0); cfma(t01, a0, b1); cfma(t10, a1, b0); cfma(t11, a1, b1);
      }
      for (int IJ = 0; IJ < 4; ++IJ) {
        cplx v = cmul(G[IJ * 4 + 0], t00);
        v = cadd(v, cmul(G[IJ * 4 + 1], t01));
        v = cadd(v, cmul(G[IJ * 4 + 2], t10));
        v = cadd(v, cmul(G[IJ * 4 + 3], t11));
        const int I = IJ >> 1, J = IJ & 1;
        if (tall) X[(J * dr + r) * 32 + (l * 2 + I)] = v;
        else X[(l * 2 + I) * 32 + (J * dr + r)] = v;
      }
    }
    // V = identity (stored transposed: VT[col][row])
    for (int e = tid; e < 32 * 32; e += NT)
      VT[e] = cmake((e >> 5) == (e & 31) ? 1.0 : 0.0, 0.0);
    __syncthreads();
    // row norms, then ||Theta||_F^2 as their sum in row order (the same bits
    // for every thread count)
    jacobi_row_norms<NT>(X, NORM, mr, mc, tid);
    __syncthreads();
    double total = 0.0;
    for (int w = 0; w < mr; ++w) total += NORM[w];
    // Rows below eps * ||Theta||_F are numerically null: pairs whose coupling
    // |gamma| is below eps^2 ||Theta||_F^2 are left alone, which keeps a
    // rank-deficient Theta from rotating rounding noise forever.
    const double floor_g = eps * eps * total;
    const double floor2 = floor_g * floor_g;
    const double tol2 = 16.0 * eps * eps;        // |gamma| > 4 eps sqrt(alpha beta)
    __syncthreads();

    // ---- one-sided Jacobi on the rows of Theta, round-robin pair ordering ----
    // A pair (p, q) with alpha = |X_p|^2, beta = |X_q|^2, gamma = X_p . X_q^H is
    // rotated by J = c [[1, -w gamma], [w conj(gamma), 1]] with
    // w = 2 sign(d) / (|d| + r), r = sqrt(d^2 + 4 |gamma|^2), d = beta - alpha,
    // c = 1 / sqrt(1 + w^2 |gamma|^2): the classical Jacobi rotation with the
    // phase of gamma moved onto row q (V absorbs it). Without a division:
    // 1 + w^2 |gamma|^2 = 2 r / (|d| + r), so with s = 1 / sqrt(r (|d| + r)),
    // w c = sign(d) sqrt(2) s, c = (|d| + r) s / sqrt(2) and
    // w |gamma|^2 = sign(d) 2 |gamma|^2 r s^2. Row norms move by -+ w |gamma|^2
    // and are kept in NORM, recomputed exactly after each sweep.
    const int grp = tid >> 4, lane = tid & 15;
    const int npairs = mr >> 1, plim = (npairs + 1) & ~1;
    // round-robin pairs of every step of a sweep (row 0 fixed, rows 1 .. mr-1 rotating)
    for (int e = tid; e < (mr - 1) * 16; e += NT) {
      const int step = e >> 4, pr_ = e & 15, mm1 = mr - 1;
      int a = 0, b = 0;
      if (pr_ < npairs) {
        if (pr_ == 0) { a = 0; b = 1 + (step % mm1); }
        else { a = 1 + ((step + pr_) % mm1); b = 1 + ((step + mm1 - pr_) % mm1); }
        if (a > b) { const int t = a; a = b; b = t; }
      }
      SCHED[e] = a | (b << 8);
    }
    __syncthreads();
    // Converged once mr - 1 consecutive steps rotate nothing: such a window
    // visits every pair exactly once (across a sweep boundary too), each with no
    // rotation since -- half a sweep earlier on average than waiting for a whole
    // quiet sweep.
    bool converged = false;
    int quiet = 0;
    for (int sweep = 0; sweep < JACOBI_MAX_SWEEPS && !converged; ++sweep) {
      for (int step = 0; step < mr - 1; ++step) {
        int rotated = 0;
        // pairs grp, grp + NT/16, ... of the step (one pass when NT = 256); the
        // pairs of a step touch disjoint rows, so their order does not matter.
        // The bound is even, so both 16-lane groups of a warp take the same
        // passes (the shuffles below need the whole warp).
        for (int pair = grp; pair < plim; pair += NT / 16) {
          const bool active = pair < npairs;
          const int pq = SCHED[step * 16 + pair];
          const int pr = pq & 255, qr = pq >> 8;
          cplx xp0 = cmake(0, 0), xq0 = cmake(0, 0), xp1 = cmake(0, 0), xq1 = cmake(0, 0);
          const int j0 = lane, j1 = lane + 16;
          if (active) {
            if (j0 < mc) { xp0 = X[pr * 32 + j0]; xq0 = X[qr * 32 + j0]; }
            if (j1 < mc) { xp1 = X[pr * 32 + j1]; xq1 = X[qr * 32 + j1]; }
          }
          // gamma = sum_j X[p,j] conj(X[q,j])
          double gr = xp0.x * xq0.x + xp0.y * xq0.y + xp1.x * xq1.x + xp1.y * xq1.y;
          double gim = xp0.y * xq0.x - xp0.x * xq0.y + xp1.y * xq1.x - xp1.x * xq1.y;
          for (int o = 8; o > 0; o >>= 1) {
            gr += __shfl_xor_sync(0xffffffffu, gr, o, 16);
            gim += __shfl_xor_sync(0xffffffffu, gim, o, 16);
          }
          const double al = active ? NORM[pr] : 0.0, be = active ? NORM[qr] : 0.0;
          const double g2 = gr * gr + gim * gim;
          if (active && g2 > floor2 && g2 > tol2 * al * be) {
            rotated = 1;
            const double d = be - al, ad = fabs(d);
            const double r = sqrt(d * d + 4.0 * g2);
            const double sr = rsqrt(r * (ad + r));
            const double wc = copysign(1.4142135623730951 * sr, d);   // w c
            const double c = (ad + r) * sr * 0.7071067811865476;
            const double wg2 = copysign(2.0 * g2 * r * sr * sr, d);    // w |gamma|^2
            const cplx wg = cmake(wc * gr, wc * gim);           // w c gamma
            const cplx wgc = cconj(wg);                         // w c conj(gamma)
            if (j0 < mc) {
              X[pr * 32 + j0] = csub(cscale(xp0, c), cmul(wg, xq0));
              X[qr * 32 + j0] = cadd(cmul(wgc, xp0), cscale(xq0, c));
            }
            if (j1 < mc) {
              X[pr * 32 + j1] = csub(cscale(xp1, c), cmul(wg, xq1));
              X[qr * 32 + j1] = cadd(cmul(wgc, xp1), cscale(xq1, c));
            }
            // V <- V J^H: V_p' = c V_p - w c conj(gamma) V_q, V_q' = w c gamma V_p + c V_q
            for (int i = lane; i < mr; i += 16) {
              const cplx vp = VT[pr * 32 + i], vq = VT[qr * 32 + i];
              VT[pr * 32 + i] = csub(cscale(vp, c), cmul(wgc, vq));
              VT[qr * 32 + i] = cadd(cmul(wg, vp), cscale(vq, c));
            }
            if (lane == 0) {
              NORM[pr] = al - wg2;
              NORM[qr] = be + wg2;
            }
          }
        }
        quiet = __syncthreads_or(rotated) ? 0 : quiet + 1;
        if (quiet >= mr - 1) {
          converged = true;
          break;
        }
      }
      jacobi_row_norms<NT>(X, NORM, mr, mc, tid);
      __syncthreads();
    }
    // ---- singular values = row norms, sorted descending (stable in row index) ----
    if (tid < mr) NORM[tid] = sqrt(NORM[tid]);
    __syncthreads();
    if (tid < mr) {
      const double v = NORM[tid];
      int rank = 0;
      for (int q = 0; q < mr; ++q) {
        const double w = NORM[q];
        rank += (w > v) || (w == v && q < tid);
      }
      PERM[rank] = tid;
      SIG[rank] = v;
    }
    __syncthreads();
    // ---- selectDirectSvdRank (dist_svd.cuh:194-212) ----
    if (tid == 0) {
      const int r = mr;                          // min(m, ncol)
      int st = converged ? ST_OK : ST_NONFINITE;
      int selected = 0;
      const double thr = fmax(p.abs_cut, p.rel_cut * SIG[0]);
      const bool zero_cut = (p.abs_cut == 0.0 && p.rel_cut == 0.0);
      for (int i = 0; i < mr; ++i)
        if (!isfinite(NORM[i])) st = ST_NONFINITE;
      for (int i = 0; i < r; ++i)
        if (zero_cut || SIG[i] > thr) ++selected;
      if (st == ST_OK && zero_cut && p.max_bond < r &&
          SIG[p.max_bond] > 64.0 * eps * r * SIG[0])
        st = ST_INSUFFICIENT;
      int k = selected < p.max_bond ? selected : p.max_bond;
      if (k < 1) k = 1;
      MISC[0] = st;
      MISC[1] = k;
    }
    __syncthreads();
    if (MISC[0] != ST_OK) return MISC[0];
    const int k = MISC[1];
    // ---- pack (packDirectSvdFactors: left = U_k (Dl,2,k), right = S_k Vh_k (k,2,Dr);
    //      with sigma_left: left = U_k S_k, right = Vh_k) ----
    // Wide Theta: Theta = V X. Tall Theta: Theta^T = V X, so Theta = X^T V^T. In
    // both, V is unitary and the rows of X are orthogonal with norms sigma, so one
    // factor is read from V (scaled by sigma when it carries them) and the other
    // from the rows of X, which are normalised when they must form the isometric
    // factor (wide with sigma_left, tall without).
    cplx *ga = sites_b + (size_t)s * SITE_ELEMS;
    cplx *gb = ga + SITE_ELEMS;
    if (tall == sigma_left) {
      // left from X's rows as they are (tall, sigma_left: U S) or from V (wide: U),
      // right from V (tall: Vh) or from X's rows (wide: S Vh)
      for (int e = tid; e < SITE_ELEMS; e += NT) {
        const int l = e >> 5, I = (e >> 4) & 1, c = e & 15;
        const int cc = e >> 5, J = (e >> 4) & 1, r = e & 15;
        if (tall) {
          ga[e] = (l < dl && c < k) ? X[PERM[c] * 32 + (l * 2 + I)] : cmake(0, 0);
          gb[e] = (cc < k && r < dr) ? VT[PERM[cc] * 32 + (J * dr + r)] : cmake(0, 0);
        } else {
          ga[e] = (l < dl && c < k) ? VT[PERM[c] * 32 + (l * 2 + I)] : cmake(0, 0);
          gb[e] = (cc < k && r < dr) ? X[PERM[cc] * 32 + (J * dr + r)] : cmake(0, 0);
        }
      }
    } else {
      // The isometric factor is X's rows divided by sigma (length mc). Rows whose
      // sigma is numerically zero (<= 64 eps r sigma_0, the rank guard's scale)
      // carry no weight; they are replaced by unit vectors made orthogonal to the
      // kept rows (two Gram-Schmidt passes), so the factor stays an isometry, as
      // gesvd's orthonormal completion does in the reference.
      cplx *UC = SA;                                   // k x mc, UC[c * 32 + i]
      const double tiny = 64.0 * eps * mr * SIG[0];
      for (int e = tid; e < k * 32; e += NT) {
        const int c = e >> 5, i = e & 31;
        UC[e] = (i < mc && SIG[c] > tiny) ? cscale(X[PERM[c] * 32 + i], 1.0 / SIG[c]) : cmake(0, 0);
      }
      __syncthreads();
      if (!(SIG[k - 1] > tiny) && tid < 32) {
        for (int c = 0; c < k; ++c) {
          if (SIG[c] > tiny) continue;
          for (int i0 = 0; i0 < mc; ++i0) {
            cplx v = cmake(tid == i0 ? 1.0 : 0.0, 0.0);
            for (int pass = 0; pass < 2; ++pass)
              for (int i = 0; i < c; ++i) {
                const cplx u = tid < mc ? UC[i * 32 + tid] : cmake(0, 0);
                double dr_ = u.x * v.x + u.y * v.y, di = u.x * v.y - u.y * v.x;   // conj(u) v
                for (int o = 16; o > 0; o >>= 1) {
                  dr_ += __shfl_xor_sync(0xffffffffu, dr_, o);
                  di += __shfl_xor_sync(0xffffffffu, di, o);
                }
                v = csub(v, cmul(cmake(dr_, di), u));
              }
            double nn = cabs2(v);
            for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
            // some basis vector keeps at least the average residual (mc - c) / mc
            if (nn > 0.5 * (double)(mc - c) / mc) {
              if (tid < mc) UC[c * 32 + tid] = cscale(v, 1.0 / sqrt(nn));
              __syncwarp();
              break;
            }
          }
        }
      }
      __syncthreads();
      for (int e = tid; e < SITE_ELEMS; e += NT) {
        const int l = e >> 5, I = (e >> 4) & 1, c = e & 15;
        const int cc = e >> 5, J = (e >> 4) & 1, r = e & 15;
        if (tall) {
          ga[e] = (l < dl && c < k) ? UC[c * 32 + (l * 2 + I)] : cmake(0, 0);
          gb[e] = (cc < k && r < dr) ? cscale(VT[PERM[cc] * 32 + (J * dr + r)], SIG[cc]) : cmake(0, 0);
        } else {
          ga[e] = (l < dl && c < k) ? cscale(VT[PERM[c] * 32 + (l * 2 + I)], SIG[c]) : cmake(0, 0);
          gb[e] = (cc < k && r < dr) ? UC[cc * 32 + (J * dr + r)] : cmake(0, 0);
        }
      }
    }
    if (tid == 0) *bond_next = k;
    __syncthreads();
    return ST_OK;
}

// NORM[row] = sum_j X[row][j]^2 for real rows (as jacobi_row_norms).
template <int NT>
__device__ __forceinline__ void jacobi_row_norms_real(const double *X, double *NORM, int mr, int mc, int tid) {
  const int grp = tid >> 4, lane = tid & 15;
  for (int row = grp; row < mr; row += NT / 16) {
    double a = 0.0;
    for (int j = lane; j < mc; j += 16) a += X[row * 32 + j] * X[row * 32 + j];
    for (int o = 8; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o, 16);
    if (lane == 0) NORM[row] = a;
  }
}

// The two-site update of two_site_update for a circuit of real gates: every
// site tensor, gate and pending one-site matrix is real (imaginary parts zero),
// so Theta, the Jacobi rotations and both factors are real and the same steps
// run in real arithmetic: the coupling gamma = X_p . X_q is a real dot product,
// the rotation J = c [[1, -w gamma], [w gamma, 1]] a Givens rotation (same
// division-free formulas with |gamma|^2 = gamma^2), and each element update two
// real multiply-adds instead of eight. The shared tiles are the complex
// function's, used as doubles; site tensors stay complex in global memory
// (written with zero imaginary parts). Rank rule, guard, ordering, packing
// (including sigma_left) and the null-direction completion are the same.
template <int NT>
__device__ __forceinline__ int two_site_update_real(const EvolveParams &p, const EvolveShared &sh, cplx *sites_b,
                                                    int s, int dl, int dc, int dr, cplx *us, cplx *ut,
                                                    const cplx *gm, int *bond_next, bool sigma_left) {
  double *X = reinterpret_cast<double *>(sh.X), *VT = reinterpret_cast<double *>(sh.VT);
  double *SA = reinterpret_cast<double *>(sh.SA), *SB = reinterpret_cast<double *>(sh.SB);
  double *G = reinterpret_cast<double *>(sh.G);
  double *NORM = sh.NORM, *SIG = sh.SIG;
  int *PERM = sh.PERM, *MISC = sh.MISC, *SCHED = sh.SCHED;
  const int tid = threadIdx.x;
  const double eps = 2.2204460492503131e-16;
  const int m = 2 * dl, ncol = 2 * dr;
  const bool tall = m > ncol;
  const int mr = tall ? ncol : m, mc = tall ? m : ncol;
  {
    const cplx *ga = sites_b + (size_t)s * SITE_ELEMS;
    const cplx *gb = ga + SITE_ELEMS;
    for (int e = tid; e < SITE_ELEMS; e += NT) { SA[e] = __ldcg(ga + e).x; SB[e] = __ldcg(gb + e).x; }
    if (tid < 16) {
      // G' = G (U_s (x) U_{s+1})
      const int row = tid >> 2, col = tid & 3;
      const int i = col >> 1, j = col & 1;
      double acc = 0.0;
      for (int ip = 0; ip < 2; ++ip)
        for (int jp = 0; jp < 2; ++jp) acc += gm[row * 4 + ip * 2 + jp].x * (us[ip * 2 + i].x * ut[jp * 2 + j].x);
      G[tid] = acc;
    }
  }
  __syncthreads();
  if (tid < 4) {
    us[tid] = cmake(tid == 0 || tid == 3 ? 1 : 0, 0);
    ut[tid] = cmake(tid == 0 || tid == 3 ? 1 : 0, 0);
  }
  // Theta[(l*2+I), (J*dr+r)] = sum_ij G'[(I*2+J)*4+(i*2+j)] sum_c A[l,i,c] B[c,j,r]
  for (int lr = tid; lr < dl * dr; lr += NT) {
    const int l = lr / dr, r = lr % dr;
    double t00 = 0.0, t01 = 0.0, t10 = 0.0, t11 = 0.0;
    for (int c = 0; c < dc; ++c) {
      const double a0 = SA[(l * 2 + 0) * CHI + c], a1 = SA[(l * 2 + 1) * CHI + c];
      const double b0 = SB[(c * 2 + 0) * CHI + r], b1 = SB[(c * 2 + 1) * CHI + r];
      t00 = fma(a0, b0, t00); t01 = fma(a0, b1, t01); t10 = fma(a1, b0, t10); t11 = fma(a1, b1, t11);
    }
    for (int IJ = 0; IJ < 4; ++IJ) {
      double v = G[IJ * 4 + 0] * t00;
      v = fma(G[IJ * 4 + 1], t01, v);
      v = fma(G[IJ * 4 + 2], t10, v);
      v = fma(G[IJ * 4 + 3], t11, v);
      const int I = IJ >> 1, J = IJ & 1;
      if (tall) X[(J * dr + r) * 32 + (l * 2 + I)] = v;
      else X[(l * 2 + I) * 32 + (J * dr + r)] = v;
    }
  }
  for (int e = tid; e < 32 * 32; e += NT) VT[e] = (e >> 5) == (e & 31) ? 1.0 : 0.0;
  __syncthreads();
  jacobi_row_norms_real<NT>(X, NORM, mr, mc, tid);
  __syncthreads();
  double total = 0.0;
  for (int w = 0; w < mr; ++w) total += NORM[w];
  const double floor_g = eps * eps * total;
  const double floor2 = floor_g * floor_g;
  const double tol2 = 16.0 * eps * eps;
  __syncthreads();
  const int grp = tid >> 4, lane = tid & 15;
  const int npairs = mr >> 1, plim = (npairs + 1) & ~1;
  for (int e = tid; e < (mr - 1) * 16; e += NT) {
    const int step = e >> 4, pr_ = e & 15, mm1 = mr - 1;
    int a = 0, b = 0;
    if (pr_ < npairs) {
      if (pr_ == 0) { a = 0; b = 1 + (step % mm1); }
      else { a = 1 + ((step + pr_) % mm1); b = 1 + ((step + mm1 - pr_) % mm1); }
      if (a > b) { const int t = a; a = b; b = t; }
    }
    SCHED[e] = a | (b << 8);
  }
  __syncthreads();
  bool converged = false;
  int quiet = 0;   // consecutive steps without a rotation (see two_site_update)
  for (int sweep = 0; sweep < JACOBI_MAX_SWEEPS && !converged; ++sweep) {
    for (int step = 0; step < mr - 1; ++step) {
      int rotated = 0;
      for (int pair = grp; pair < plim; pair += NT / 16) {
        const bool active = pair < npairs;
        const int pq = SCHED[step * 16 + pair];
        const int pr = pq & 255, qr = pq >> 8;
        double xp0 = 0.0, xq0 = 0.0, xp1 = 0.0, xq1 = 0.0;
        const int j0 = lane, j1 = lane + 16;
        if (active) {
          if (j0 < mc) { xp0 = X[pr * 32 + j0]; xq0 = X[qr * 32 + j0]; }
          if (j1 < mc) { xp1 = X[pr * 32 + j1]; xq1 = X[qr * 32 + j1]; }
        }
        double gr = fma(xp1, xq1, xp0 * xq0);
        for (int o = 8; o > 0; o >>= 1) gr += __shfl_xor_sync(0xffffffffu, gr, o, 16);
        const double al = active ? NORM[pr] : 0.0, be = active ? NORM[qr] : 0.0;
        const double g2 = gr * gr;
        if (active && g2 > floor2 && g2 > tol2 * al * be) {
          rotated = 1;
          const double d = be - al, ad = fabs(d);
          const double r = sqrt(d * d + 4.0 * g2);
          const double sr = rsqrt(r * (ad + r));
          const double wc = copysign(1.4142135623730951 * sr, d);   // w c
          const double c = (ad + r) * sr * 0.7071067811865476;
          const double wg2 = copysign(2.0 * g2 * r * sr * sr, d);    // w gamma^2
          const double wg = wc * gr;                                  // w c gamma
          if (j0 < mc) {
            X[pr * 32 + j0] = fma(c, xp0, -wg * xq0);
            X[qr * 32 + j0] = fma(wg, xp0, c * xq0);
          }
          if (j1 < mc) {
            X[pr * 32 + j1] = fma(c, xp1, -wg * xq1);
            X[qr * 32 + j1] = fma(wg, xp1, c * xq1);
          }
          for (int i = lane; i < mr; i += 16) {
            const double vp = VT[pr * 32 + i], vq = VT[qr * 32 + i];
            VT[pr * 32 + i] = fma(c, vp, -wg * vq);
            VT[qr * 32 + i] = fma(wg, vp, c * vq);
          }
          if (lane == 0) {
            NORM[pr] = al - wg2;
            NORM[qr] = be + wg2;
          }
        }
      }
      quiet = __syncthreads_or(rotated) ? 0 : quiet + 1;
      if (quiet >= mr - 1) {
        converged = true;
        break;
      }
    }
    jacobi_row_norms_real<NT>(X, NORM, mr, mc, tid);
    __syncthreads();
  }
  if (tid < mr) NORM[tid] = sqrt(NORM[tid]);
  __syncthreads();
  if (tid < mr) {
    const double v = NORM[tid];
    int rank = 0;
    for (int q = 0; q < mr; ++q) {
      const double w = NORM[q];
      rank += (w > v) || (w == v && q < tid);
    }
    PERM[rank] = tid;
    SIG[rank] = v;
  }
  __syncthreads();
  if (tid == 0) {
    const int r = mr;
    int st = converged ? ST_OK : ST_NONFINITE;
    int selected = 0;
    const double thr = fmax(p.abs_cut, p.rel_cut * SIG[0]);
    const bool zero_cut = (p.abs_cut == 0.0 && p.rel_cut == 0.0);
    for (int i = 0; i < mr; ++i)
      if (!isfinite(NORM[i])) st = ST_NONFINITE;
    for (int i = 0; i < r; ++i)
      if (zero_cut || SIG[i] > thr) ++selected;
    if (st == ST_OK && zero_cut && p.max_bond < r && SIG[p.max_bond] > 64.0 * eps * r * SIG[0])
      st = ST_INSUFFICIENT;
    int k = selected < p.max_bond ? selected : p.max_bond;
    if (k < 1) k = 1;
    MISC[0] = st;
    MISC[1] = k;
  }
  __syncthreads();
  if (MISC[0] != ST_OK) return MISC[0];
  const int k = MISC[1];
  cplx *ga = sites_b + (size_t)s * SITE_ELEMS;
  cplx *gb = ga + SITE_ELEMS;
  if (tall == sigma_left) {
    for (int e = tid; e < SITE_ELEMS; e += NT) {
      const int l = e >> 5, I = (e >> 4) & 1, c = e & 15;
      const int cc = e >> 5, J = (e >> 4) & 1, r = e & 15;
      double va, vb;
      if (tall) {
        va = (l < dl && c < k) ? X[PERM[c] * 32 + (l * 2 + I)] : 0.0;
        vb = (cc < k && r < dr) ? VT[PERM[cc] * 32 + (J * dr + r)] : 0.0;
      } else {
        va = (l < dl && c < k) ? VT[PERM[c] * 32 + (l * 2 + I)] : 0.0;
        vb = (cc < k && r < dr) ? X[PERM[cc] * 32 + (J * dr + r)] : 0.0;
      }
      ga[e] = cmake(va, 0.0);
      gb[e] = cmake(vb, 0.0);
    }
  } else {
    double *UC = SA;                                 // k x mc, UC[c * 32 + i]
    const double tiny = 64.0 * eps * mr * SIG[0];
    for (int e = tid; e < k * 32; e += NT) {
      const int c = e >> 5, i = e & 31;
      UC[e] = (i < mc && SIG[c] > tiny) ? X[PERM[c] * 32 + i] * (1.0 / SIG[c]) : 0.0;
    }
    __syncthreads();
    if (!(SIG[k - 1] > tiny) && tid < 32) {
      for (int c = 0; c < k; ++c) {
        if (SIG[c] > tiny) continue;
        for (int i0 = 0; i0 < mc; ++i0) {
          double v = tid == i0 ? 1.0 : 0.0;
          for (int pass = 0; pass < 2; ++pass)
            for (int i = 0; i < c; ++i) {
              const double u = tid < mc ? UC[i * 32 + tid] : 0.0;
              double dt = u * v;
              for (int o = 16; o > 0; o >>= 1) dt += __shfl_xor_sync(0xffffffffu, dt, o);
              v -= dt * u;
            }
          double nn = v * v;
          for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xffffffffu, nn, o);
          if (nn > 0.5 * (double)(mc - c) / mc) {
            if (tid < mc) UC[c * 32 + tid] = v * (1.0 / sqrt(nn));
            __syncwarp();
            break;
          }
        }
      }
    }
    __syncthreads();
    for (int e = tid; e < SITE_ELEMS; e += NT) {
      const int l = e >> 5, I = (e >> 4) & 1, c = e & 15;
      const int cc = e >> 5, J = (e >> 4) & 1, r = e & 15;
      double va, vb;
      if (tall) {
        va = (l < dl && c < k) ? UC[c * 32 + (l * 2 + I)] : 0.0;
        vb = (cc < k && r < dr) ? VT[PERM[cc] * 32 + (J * dr + r)] * SIG[cc] : 0.0;
      } else {
        va = (l < dl && c < k) ? VT[PERM[c] * 32 + (l * 2 + I)] * SIG[c] : 0.0;
        vb = (cc < k && r < dr) ? UC[cc * 32 + (J * dr + r)] : 0.0;
      }
      ga[e] = cmake(va, 0.0);
      gb[e] = cmake(vb, 0.0);
    }
  }
  if (tid == 0) *bond_next = k;
  __syncthreads();
  return ST_OK;
}

// Chain arithmetic: complex, real (a circuit of real gates), or chosen per
// partition of a mixed partition set (EvolveParams::part_real).
enum : int { CHAIN_COMPLEX = 0, CHAIN_REAL = 1, CHAIN_PER_PARTITION = 2 };

template <int NT, int MODE>
__device__ __forceinline__ int gate_update(const EvolveParams &p, const EvolveShared &sh, cplx *sites_b, int s,
                                           int dl, int dc, int dr, cplx *us, cplx *ut, const cplx *gm,
                                           int *bond_next, bool sigma_left, bool part_real) {
  if constexpr (MODE == CHAIN_REAL) {
    return two_site_update_real<NT>(p, sh, sites_b, s, dl, dc, dr, us, ut, gm, bond_next, sigma_left);
  } else if constexpr (MODE == CHAIN_COMPLEX) {
    return two_site_update<NT>(p, sh, sites_b, s, dl, dc, dr, us, ut, gm, bond_next, sigma_left);
  } else {
    if (part_real) return two_site_update_real<NT>(p, sh, sites_b, s, dl, dc, dr, us, ut, gm, bond_next, sigma_left);
    return two_site_update<NT>(p, sh, sites_b, s, dl, dc, dr, us, ut, gm, bond_next, sigma_left);
  }
}

template <int MODE>
__device__ __forceinline__ void evolve_body(const EvolveParams &p) {
  extern __shared__ __align__(16) unsigned char smem[];
  cplx *X = reinterpret_cast<cplx *>(smem + EvolveSmem::X);
  cplx *VT = reinterpret_cast<cplx *>(smem + EvolveSmem::VT);
  cplx *SA = reinterpret_cast<cplx *>(smem + EvolveSmem::SA);
  cplx *SB = reinterpret_cast<cplx *>(smem + EvolveSmem::SB);
  cplx *G = reinterpret_cast<cplx *>(smem + EvolveSmem::G);
  double *NORM = reinterpret_cast<double *>(smem + EvolveSmem::NORM);
  double *SIG = reinterpret_cast<double *>(smem + EvolveSmem::SIG);
  int *PERM = reinterpret_cast<int *>(smem + EvolveSmem::PERM);
  int *MISC = reinterpret_cast<int *>(smem + EvolveSmem::MISC);
  int *SCHED = reinterpret_cast<int *>(smem + EvolveSmem::SCHED);
  cplx *PEND = reinterpret_cast<cplx *>(smem + EvolveSmem::PEND);
  int *BOND = reinterpret_cast<int *>(smem + EvolveSmem::PEND + p.n * 4 * 16);

  const int tid = threadIdx.x;
  const int b = blockIdx.x;
  const int part = p.st_part ? p.st_part[b] : 0;
  const bool part_real = MODE == CHAIN_PER_PARTITION && p.part_real[part] != 0;
  const int n = p.st_part ? p.part_n[part] : p.n;
  const int gate_begin = p.st_part ? p.part_gate_off[part] : 0;
  const int gate_end = p.st_part ? p.part_gate_off[part + 1] : p.ngates;
  const double *theta_b = p.theta + (size_t)b * p.P;
  cplx *sites_b = p.sites + (size_t)b * p.n * SITE_ELEMS;

  // |init>^n product state, zero padded; identity pending matrices.
  for (int e = tid; e < n * SITE_ELEMS; e += EVOLVE_THREADS) {
    int el = e % SITE_ELEMS;
    cplx v = cmake(0, 0);
    if (el == 0) v = p.init0;
    else if (el == CHI) v = p.init1;   // (l=0, p=1, r=0)
    sites_b[e] = v;
  }
  for (int s = tid; s < n; s += EVOLVE_THREADS) {
    PEND[s * 4 + 0] = cmake(1, 0); PEND[s * 4 + 1] = cmake(0, 0);
    PEND[s * 4 + 2] = cmake(0, 0); PEND[s * 4 + 3] = cmake(1, 0);
  }
  for (int s = tid; s <= n; s += EVOLVE_THREADS) BOND[s] = 1;
  if (tid == 0) MISC[0] = ST_OK;
  __syncthreads();

  for (int gi = gate_begin; gi < gate_end; ++gi) {
    const DevGate g = p.gates[gi];
    if (g.kind == GATE_ONE) {
      if (tid == 0) {
        cplx m[4];
        one_site_matrix(g, p.mats, theta_b, m);
        left_multiply_2x2(m, PEND + g.site * 4);
      }
      __syncthreads();
      continue;
    }
    const int s = g.site;
    const EvolveShared sh{X, VT, SA, SB, G, NORM, SIG, PERM, MISC, SCHED};
    if (gate_update<EVOLVE_THREADS, MODE>(p, sh, sites_b, s, BOND[s], BOND[s + 1], BOND[s + 2], PEND + s * 4,
                                          PEND + (s + 1) * 4, p.mats + g.mat, BOND + s + 1,
                                          (g.flags & GATE_SIGMA_LEFT) != 0, part_real) != ST_OK)
      break;
  }
  const int status = MISC[0];
  if (status == ST_OK) {
    // apply the still-pending one-site matrices in place (apply1q)
    for (int s = 0; s < n; ++s) apply_2x2_to_site(PEND + s * 4, sites_b + (size_t)s * SITE_ELEMS, tid, EVOLVE_THREADS);
  }
  for (int s = tid; s <= n; s += EVOLVE_THREADS) p.bonds[(size_t)b * (p.n + 1) + s] = BOND[s];
  if (tid == 0) p.status[b] = status;
}

__global__ void __launch_bounds__(EVOLVE_THREADS, 3)
evolve_kernel(EvolveParams p) { evolve_body<CHAIN_COMPLEX>(p); }

// The same chain for a circuit of real gates (real-arithmetic Jacobi SVD).
__global__ void __launch_bounds__(EVOLVE_THREADS, 3)
evolve_real_kernel(EvolveParams p) { evolve_body<CHAIN_REAL>(p); }

// A partition set mixing real and complex circuits: each state's arithmetic is
// its partition's, so every partition gets the one-partition engine's bits.
__global__ void __launch_bounds__(EVOLVE_THREADS, 3)
evolve_mixed_kernel(EvolveParams p) { evolve_body<CHAIN_PER_PARTITION>(p); }

// 2 x 2 product of the one-site gates qlist[q0 .. q1) in program order (later
// gates on the left).
__device__ __forceinline__ void pending_product(const EvolveParams &p, const double *theta_b, int q0, int q1,
                                                cplx *u) {
  u[0] = cmake(1, 0); u[1] = cmake(0, 0); u[2] = cmake(0, 0); u[3] = cmake(1, 0);
  for (int q = q0; q < q1; ++q) {
    cplx m[4];
    one_site_matrix(p.gates[p.qlist[q]], p.mats, theta_b, m);
    left_multiply_2x2(m, u);
  }
}

// Pending one-site products of every two-site gate and state (grid: gate blocks x
// states): one thread per gate, the same products in the same order as
// pending_product inside the chain, so the states are unchanged bit for bit.
__global__ void __launch_bounds__(128)
pending_kernel(EvolveParams p, cplx *upend) {
  const int b = blockIdx.y;
  const int gi = blockIdx.x * 128 + threadIdx.x;
  if (gi >= p.ngates) return;
  const DevGate g = p.gates[gi];
  if (g.kind != GATE_TWO) return;
  const double *theta_b = p.theta + (size_t)b * p.P;
  cplx u[8];
  pending_product(p, theta_b, p.gate_q[4 * gi + 0], p.gate_q[4 * gi + 1], u);
  pending_product(p, theta_b, p.gate_q[4 * gi + 2], p.gate_q[4 * gi + 3], u + 4);
  cplx *dst = upend + ((size_t)b * p.ngates + gi) * 8;
  for (int k = 0; k < 8; ++k) dst[k] = u[k];
}

// The gate chain of one state on a cluster of two CTAs. Two-site gates on
// disjoint site pairs commute, so a precomputed as-soon-as-possible schedule of
// at most two gates per step (one per CTA) replaces program order; each step
// ends with one cluster barrier. Every gate runs the same code on the same data
// as in evolve_kernel (pending one-site gates folded in the same order), so the
// state is bit-for-bit the sequential one. Site tensors and bond dimensions live
// in global memory (read past L1 with ld.global.cg, since the other CTA writes
// them). Both CTAs take every step, whatever the status, so the barrier counts
// always match; after a failure the remaining gates are skipped.
template <int MODE, int K, class SM>
__device__ __forceinline__ void evolve_pair_body(const EvolveParams &p) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem[];
  cplx *X = reinterpret_cast<cplx *>(smem + SM::X);
  cplx *VT = reinterpret_cast<cplx *>(smem + SM::VT);
  cplx *SA = reinterpret_cast<cplx *>(smem + SM::SA);
  cplx *SB = reinterpret_cast<cplx *>(smem + SM::SB);
  cplx *G = reinterpret_cast<cplx *>(smem + SM::G);
  double *NORM = reinterpret_cast<double *>(smem + SM::NORM);
  double *SIG = reinterpret_cast<double *>(smem + SM::SIG);
  int *PERM = reinterpret_cast<int *>(smem + SM::PERM);
  int *MISC = reinterpret_cast<int *>(smem + SM::MISC);
  int *SCHED = reinterpret_cast<int *>(smem + SM::SCHED);
  cplx *U = reinterpret_cast<cplx *>(smem + SM::PEND);     // 8 entries: U_s, U_{s+1}

  const int tid = threadIdx.x;
  const int rank = (int)cluster.block_rank();
  const int b = blockIdx.x / K;
  const int part = p.st_part ? p.st_part[b] : 0;
  const bool part_real = MODE == CHAIN_PER_PARTITION && p.part_real[part] != 0;
  const int n = p.st_part ? p.part_n[part] : p.n;
  const double *theta_b = p.theta + (size_t)b * p.P;
  cplx *sites_b = p.sites + (size_t)b * p.n * SITE_ELEMS;
  int32_t *bonds_b = p.bonds + (size_t)b * (p.n + 1);
  volatile int32_t *status_b = p.status + b;

  // |init>^n product state and unit bonds, split between the K CTAs
  for (int e = tid + rank * PAIR_THREADS; e < n * SITE_ELEMS; e += K * PAIR_THREADS) {
    const int el = e % SITE_ELEMS;
    cplx v = cmake(0, 0);
    if (el == 0) v = p.init0;
    else if (el == CHI) v = p.init1;
    sites_b[e] = v;
  }
  for (int x = tid + rank * PAIR_THREADS; x <= n; x += K * PAIR_THREADS) bonds_b[x] = 1;
  if (rank == 0 && tid == 0) *status_b = ST_OK;
  __threadfence();
  cluster.sync();

  const int t0 = p.step_off ? p.step_off[part] : 0;
  const int t1 = p.step_off ? p.step_off[part + 1] : p.nsteps;
  const EvolveShared sh{X, VT, SA, SB, G, NORM, SIG, PERM, MISC, SCHED};
  // precomputed pending products (p.upend): threads 0..7 hold the entries of this
  // CTA's gate of the next step, loaded one step ahead
  const cplx *upend_b = p.upend ? p.upend + (size_t)b * p.ngates * 8 : nullptr;
  cplx unext = cmake(0, 0);
  if (upend_b && tid < 8 && t0 < t1) {
    const int g0 = p.sched[K * t0 + rank];
    if (g0 >= 0) unext = upend_b[(size_t)g0 * 8 + tid];
  }
  for (int t = t0; t < t1; ++t) {
    const int gi = p.sched[K * t + rank];
    const cplx ucur = unext;
    if (upend_b && tid < 8 && t + 1 < t1) {
      const int gn = p.sched[K * (t + 1) + rank];
      if (gn >= 0) unext = upend_b[(size_t)gn * 8 + tid];
    }
    // the other CTA may be writing the status of this step: one vote per CTA
    const bool ok = __syncthreads_and(*status_b == ST_OK);
    if (gi >= 0 && ok) {
      const DevGate g = p.gates[gi];
      if (upend_b) {
        if (tid < 8) U[tid] = ucur;
      } else if (tid == 0) {
        pending_product(p, theta_b, p.gate_q[4 * gi + 0], p.gate_q[4 * gi + 1], U);
        pending_product(p, theta_b, p.gate_q[4 * gi + 2], p.gate_q[4 * gi + 3], U + 4);
      }
      __syncthreads();
      const int s = g.site;
      const int dl = __ldcg(bonds_b + s), dc = __ldcg(bonds_b + s + 1), dr = __ldcg(bonds_b + s + 2);
      const int st = gate_update<PAIR_THREADS, MODE>(p, sh, sites_b, s, dl, dc, dr, U, U + 4, p.mats + g.mat,
                                                     bonds_b + s + 1, (g.flags & GATE_SIGMA_LEFT) != 0, part_real);
      if (st != ST_OK && tid == 0) *status_b = st;
    }
    __threadfence();
    cluster.sync();
  }
  // one-site gates after the last two-site gate on each site (site x on CTA x mod K)
  if (__syncthreads_and(*status_b == ST_OK)) {
    const int base = p.part_tail_off ? p.part_tail_off[part] : 0;
    for (int x = rank; x < n; x += K) {
      __syncthreads();
      if (tid == 0) pending_product(p, theta_b, p.tail_off[base + x], p.tail_off[base + x + 1], U);
      __syncthreads();
      apply_2x2_to_site(U, sites_b + (size_t)x * SITE_ELEMS, tid, PAIR_THREADS);
    }
  }
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PAIR_THREADS, 4)
evolve_pair_kernel(EvolveParams p) { evolve_pair_body<CHAIN_COMPLEX, 2, EvolveSmem>(p); }

// The two-CTA chain for a circuit of real gates (real-arithmetic Jacobi SVD).
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PAIR_THREADS, 4)
evolve_pair_real_kernel(EvolveParams p) { evolve_pair_body<CHAIN_REAL, 2, EvolveSmem>(p); }

// The two-CTA chain of a mixed partition set (arithmetic per partition).
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PAIR_THREADS, 4)
evolve_pair_mixed_kernel(EvolveParams p) { evolve_pair_body<CHAIN_PER_PARTITION, 2, EvolveSmem>(p); }

// A circuit of real gates on a cluster of four CTAs: up to four gates per step
// (the layers of a nearest-neighbour ansatz overlap in a wavefront: the 40-qubit,
// 4-layer benchmark circuit takes 45 steps instead of 80 with two CTAs), on the
// compact real tiles. The engine takes it while the batch needs at most about
// four CTAs per SM (beyond that the extra resident warps only wait at the CTA
// barriers). Same gates, same code, same bits as the one-CTA chain.
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(PAIR_THREADS, 4)
evolve_quad_real_kernel(EvolveParams p) { evolve_pair_body<CHAIN_REAL, 4, EvolveSmemReal>(p); }

}  // namespace vqemps
