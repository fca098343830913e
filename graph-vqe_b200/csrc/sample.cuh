// Perfect (Ferris-Vidal) bitstring sampling and shot estimates of Z words.
//
// Reference algorithm (test/backend/source/sharded_mps.cuh):
//   prepareSamplingRightEnvironments / k_rightStage / k_rightFinish  :814-836, 61-90
//   sampleBitsFromPreparedRight / k_sampleW / k_sampleProbabilities /
//   k_chooseSample / sampleHash                                      :838-877, 103-188
//   sampleZExpectationsGpu / k_zSampleSums                           :906-935, 193-214
//   sampleZExpectationsIndependentGpu (one stream per Z word)       :942-982
//
// B200 design: one THREAD per shot walks all sites in one launch (the reference
// launches three kernels per site). A CTA owns SAMPLE_THREADS shots of one
// state; at each site it stages the site tensor and the two branch matrices
// M_i[a,a'] = sum conj(A[a,i,c]) R_{s+1}[c,c'] A[a',i,c'] in shared memory (the
// right-environment sweep produces them: R_s = M_0 + M_1), and every thread
// reads them with warp-uniform addresses (broadcast). A shot keeps only its
// left vector v in registers. Bits are packed into 64-bit words in QUBIT order;
// Z-word parities are popcounts of (bits & mask).
#pragma once
#include "common.cuh"

namespace vqemps {

__host__ __device__ __forceinline__ uint64_t splitmix_hash(uint64_t x) {
  // SplitMix64 finaliser (Steele, Lea, Flood 2014), as sampleHash.
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  // Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
    const uint32_t n3 = (uint32_t)p0;
    c[0] = n0; c[1] = n1; c[2] = n2; c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Uniform in [0, 1) for (seed, site, shot).
__device__ __forceinline__ double draw_uniform(int rng, uint64_t seed, int site, int shot) {
  if (rng == 0) {
    // reference: ((u64)seed << 32) ^ ((u64)site << 20) ^ shot, seed a 32-bit unsigned
    const uint64_t raw = splitmix_hash(((seed & 0xffffffffULL) << 32) ^
                                       ((uint64_t)site << 20) ^ (uint64_t)shot);
    return (double)(raw >> 11) * 0x1.0p-53;
  }
  uint32_t c[4] = {(uint32_t)shot, (uint32_t)site, 0u, 0u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const uint64_t bits53 = (((uint64_t)c[0] << 21) ^ ((uint64_t)c[1] >> 11)) & ((1ULL << 53) - 1);
  return (double)bits53 * 0x1.0p-53;
}

constexpr int SAMPLE_THREADS = 128;
constexpr int MAX_WORDS64 = 4;   // up to 256 qubits

struct SampleParams {
  const cplx *sites;        // B x n x SITE_ELEMS
  const cplx *branch;       // B x n x 2 x ENV_ELEMS: M_i of every site (right_env_kernel)
  const int32_t *status;    // B
  int n, shots, W;
  int site_order;           // 0: site = qubit, 1: site = n-1-qubit
  int rng;
  // shared mode: one seed per state (seeds[b]); per-word mode: seeds[b * nwords + listed word]
  const uint64_t *seeds;
  uint64_t *bits;           // shared mode: B x shots x W
  // per-word mode
  const uint64_t *zmask;    // T x W (qubit order)
  const int32_t *words;     // list of word indices to sample
  const int32_t *last_site; // per listed word: last site to sample (inclusive)
  int nwords;
  int32_t *sums;            // B x nwords
  // partition sets (null: uniform batch): width part_n[st_part[b]], stride n
  const int32_t *st_part;
  const int32_t *part_n;
};

// One thread = one shot. MODE 0: shared sample set, writes packed bits.
// MODE 1: independent stream per listed Z word, accumulates parity sums.
template <int MODE>
__global__ void __launch_bounds__(SAMPLE_THREADS)
sample_kernel(SampleParams p) {
  __shared__ cplx A[SITE_ELEMS];
  __shared__ cplx M[2 * ENV_ELEMS];
  __shared__ int red[SAMPLE_THREADS / 32];
  const int b = MODE == 0 ? blockIdx.y : blockIdx.z;
  const int widx = MODE == 0 ? 0 : blockIdx.y;
  const int shot = blockIdx.x * SAMPLE_THREADS + threadIdx.x;
  const bool live = shot < p.shots && p.status[b] == 0;
  const uint64_t seed = MODE == 0 ? p.seeds[b] : p.seeds[(size_t)b * p.nwords + widx];
  const int nb = p.st_part ? p.part_n[p.st_part[b]] : p.n;
  const int last = MODE == 0 ? nb - 1 : p.last_site[widx];
  const cplx *sb = p.sites + (size_t)b * p.n * SITE_ELEMS;

  cplx v[CHI];
#pragma unroll
  for (int a = 0; a < CHI; ++a) v[a] = cmake(a == 0 ? 1.0 : 0.0, 0.0);
  uint64_t word[MAX_WORDS64] = {0, 0, 0, 0};
  const cplx *mb = p.branch + (size_t)b * p.n * 2 * ENV_ELEMS;

  for (int s = 0; s <= last; ++s) {
    __syncthreads();
    for (int e = threadIdx.x; e < SITE_ELEMS; e += SAMPLE_THREADS) A[e] = sb[(size_t)s * SITE_ELEMS + e];
    for (int e = threadIdx.x; e < 2 * ENV_ELEMS; e += SAMPLE_THREADS) M[e] = mb[(size_t)s * 2 * ENV_ELEMS + e];
    __syncthreads();
    // p_i = Re v^H M_i v with M_i[a,a'] = sum conj(A[a,i,c]) R_{s+1}[c,c'] A[a',i,c'],
    // the same number as Re(w_i^H R w_i), w_i = v A_i (k_sampleProbabilities)
    double p0 = 0.0, p1 = 0.0;
#pragma unroll
    for (int a = 0; a < CHI; ++a) {
      cplx y0 = cmake(0, 0), y1 = cmake(0, 0);
#pragma unroll
      for (int ap = 0; ap < CHI; ++ap) {
        cfma(y0, M[a * CHI + ap], v[ap]);
        cfma(y1, M[ENV_ELEMS + a * CHI + ap], v[ap]);
      }
      p0 += v[a].x * y0.x + v[a].y * y0.y;
      p1 += v[a].x * y1.x + v[a].y * y1.y;
    }
    p0 = p0 > 0.0 ? p0 : 0.0;
    p1 = p1 > 0.0 ? p1 : 0.0;
    double tot = p0 + p1;
    if (tot <= 0.0) { p0 = p1 = 0.5; tot = 1.0; }
    // k_chooseSample
    const double u = draw_uniform(p.rng, seed, s, shot);
    const int sel = u < p0 / tot ? 0 : 1;
    const double ps = sel ? p1 : p0;
    const double inv = ps > 0.0 ? 1.0 / sqrt(ps) : 1.0;
    // v <- (v A_sel) / sqrt(p_sel)
    cplx w[CHI];
#pragma unroll
    for (int c = 0; c < CHI; ++c) w[c] = cmake(0, 0);
#pragma unroll
    for (int a = 0; a < CHI; ++a)
#pragma unroll
      for (int c = 0; c < CHI; ++c) cfma(w[c], v[a], A[(a * 2 + sel) * CHI + c]);
#pragma unroll
    for (int c = 0; c < CHI; ++c) v[c] = cscale(w[c], inv);
    const int q = p.site_order == 1 ? nb - 1 - s : s;
    if (sel) word[q >> 6] |= (1ULL << (q & 63));
  }
  if (MODE == 0) {
    if (live) {
      uint64_t *dst = p.bits + ((size_t)b * p.shots + shot) * p.W;
      for (int w = 0; w < p.W; ++w) dst[w] = word[w];
    }
  } else {
    int parity = 0;
    const uint64_t *mask = p.zmask + (size_t)p.words[widx] * p.W;
    for (int w = 0; w < p.W; ++w) parity ^= __popcll(word[w] & mask[w]) & 1;
    int val = live ? (parity ? -1 : 1) : 0;
    for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = val;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < SAMPLE_THREADS / 32; ++w) t += red[w];
      atomicAdd(p.sums + (size_t)b * p.nwords + widx, t);
    }
  }
}

// sums[b, t] = sum over shots of (-1)^popc(bits & zmask[t]) for every word t.
constexpr int ZSUM_THREADS = 256;
constexpr int ZSUM_CHUNK = 512;
__global__ void __launch_bounds__(ZSUM_THREADS)
zsum_kernel(const uint64_t *__restrict__ bits, int shots, int W, const uint64_t *__restrict__ zmask,
            int T, int32_t *__restrict__ sums) {
  __shared__ uint64_t sh[ZSUM_CHUNK * MAX_WORDS64];
  const int b = blockIdx.y;
  const int t = blockIdx.x * ZSUM_THREADS + threadIdx.x;
  uint64_t m[MAX_WORDS64] = {0, 0, 0, 0};
  if (t < T)
    for (int w = 0; w < W; ++w) m[w] = zmask[(size_t)t * W + w];
  int acc = 0;
  const uint64_t *bb = bits + (size_t)b * shots * W;
  for (int base = 0; base < shots; base += ZSUM_CHUNK) {
    const int cnt = min(ZSUM_CHUNK, shots - base);
    __syncthreads();
    for (int e = threadIdx.x; e < cnt * W; e += ZSUM_THREADS) sh[e] = bb[(size_t)base * W + e];
    __syncthreads();
    if (t < T) {
      for (int k = 0; k < cnt; ++k) {
        int par = 0;
        for (int w = 0; w < W; ++w) par ^= __popcll(sh[k * W + w] & m[w]);
        acc += (par & 1) ? -1 : 1;
      }
    }
  }
  if (t < T) sums[(size_t)b * T + t] = acc;
}

// Partition sets: state b uses the part_T[k] masks of partition k = st_part[b]
// (zmask rows k * term_stride ..) and writes sums[b * term_stride + t].
__global__ void __launch_bounds__(ZSUM_THREADS)
zsum_multi_kernel(const uint64_t *__restrict__ bits, int shots, int W, const uint64_t *__restrict__ zmask,
                  int term_stride, const int32_t *__restrict__ st_part, const int32_t *__restrict__ part_T,
                  int32_t *__restrict__ sums) {
  __shared__ uint64_t sh[ZSUM_CHUNK * MAX_WORDS64];
  const int b = blockIdx.y;
  const int k = st_part[b];
  const int T = part_T[k];
  if (blockIdx.x * ZSUM_THREADS >= T) return;
  const int t = blockIdx.x * ZSUM_THREADS + threadIdx.x;
  uint64_t m[MAX_WORDS64] = {0, 0, 0, 0};
  if (t < T)
    for (int w = 0; w < W; ++w) m[w] = zmask[((size_t)k * term_stride + t) * W + w];
  int acc = 0;
  const uint64_t *bb = bits + (size_t)b * shots * W;
  for (int base = 0; base < shots; base += ZSUM_CHUNK) {
    const int cnt = min(ZSUM_CHUNK, shots - base);
    __syncthreads();
    for (int e = threadIdx.x; e < cnt * W; e += ZSUM_THREADS) sh[e] = bb[(size_t)base * W + e];
    __syncthreads();
    if (t < T) {
      for (int kk = 0; kk < cnt; ++kk) {
        int par = 0;
        for (int w = 0; w < W; ++w) par ^= __popcll(sh[kk * W + w] & m[w]);
        acc += (par & 1) ? -1 : 1;
      }
    }
  }
  if (t < T) sums[(size_t)b * term_stride + t] = acc;
}

// Shot-estimated energies: value_t = sums[t] / shots for sampled words, the
// analytic per-term value for the others; fixed-order reduction per state.
__device__ __forceinline__ void sampled_energy_body(const int32_t *__restrict__ sums,
                                                    const int32_t *__restrict__ sum_index,
                                                    const double *__restrict__ analytic,
                                                    const double *__restrict__ coeffs, int T, int shots, bool ok,
                                                    double *__restrict__ energy, double *__restrict__ per_term) {
  __shared__ double part[REDUCE_THREADS];
  const int tid = threadIdx.x;
  double acc = 0.0;
  for (int t = tid; t < T; t += REDUCE_THREADS) {
    const int si = sum_index[t];
    // si >= 0: sampled word; -2: identity word (+1 on every shot); -1: analytic (X/Y)
    const double v = si >= 0 ? (double)sums[si] / shots : (si == -2 ? 1.0 : analytic[t]);
    if (per_term) per_term[t] = ok ? v : __longlong_as_double(0x7ff8000000000000LL);
    acc = fma(coeffs[t], v, acc);
  }
  part[tid] = acc;
  __syncthreads();
  for (int w = REDUCE_THREADS / 2; w > 0; w >>= 1) {
    if (tid < w) part[tid] += part[tid + w];
    __syncthreads();
  }
  if (tid == 0) *energy = ok ? part[0] : __longlong_as_double(0x7ff8000000000000LL);
}

__global__ void __launch_bounds__(REDUCE_THREADS)
sampled_energy_kernel(const int32_t *__restrict__ sums, int sums_stride, const int32_t *__restrict__ sum_index,
                      const double *__restrict__ analytic, const double *__restrict__ coeffs, int T, int shots,
                      const int32_t *__restrict__ status, double *__restrict__ energies,
                      double *__restrict__ per_term) {
  const int b = blockIdx.x;
  sampled_energy_body(sums + (size_t)b * sums_stride, sum_index, analytic ? analytic + (size_t)b * T : nullptr,
                      coeffs, T, shots, status[b] == 0, energies + b,
                      per_term ? per_term + (size_t)b * T : nullptr);
}

// Partition sets: every array is strided by term_stride, per partition
// (sum_index, coeffs) or per state (sums, analytic, per_term).
__global__ void __launch_bounds__(REDUCE_THREADS)
sampled_energy_multi_kernel(const int32_t *__restrict__ sums, const int32_t *__restrict__ sum_index,
                            const double *__restrict__ analytic, const double *__restrict__ coeffs,
                            int term_stride, const int32_t *__restrict__ st_part,
                            const int32_t *__restrict__ part_T, int shots, const int32_t *__restrict__ status,
                            double *__restrict__ energies, double *__restrict__ per_term) {
  const int b = blockIdx.x;
  const int k = st_part[b];
  const size_t so = (size_t)b * term_stride, po = (size_t)k * term_stride;
  sampled_energy_body(sums + so, sum_index + po, analytic ? analytic + so : nullptr, coeffs + po, part_T[k],
                      shots, status[b] == 0, energies + b, per_term ? per_term + so : nullptr);
}

}  // namespace vqemps
