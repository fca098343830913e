// Message-passing network of the learned warm start: forward, backward and
// Adam, hand-written for sm_100a.
//
// No reference counterpart: the reference's warm start is the plain partition
// heuristic (test/sources/independent-vqe/Qiskit_VQE/independent_vqe.py:140-158,
// 257-305). This network reads the Hamiltonian's qubit-coupling graph and
// proposes the ansatz angles; the engine's exact MPS energy judges every
// proposal, and the partition warm start stays the fallback.
//
// Network (width W = 128, L = 3 layers, out = angles per qubit):
//   X0 = relu(F Win + bin)                                   F: N x node_in
//   per layer l:  M = relu([X[src] | Fe] Wm + bm)            per directed edge
//                 A[i] = mean over edges into i of M
//                 R = relu([X | A] Wu + bu);  X <- X + R      residual update
//   Z = X Wo + bo;  theta = pi * tanh(Z)
//
// Every matrix product runs on the tensor cores as mma.sync m16n8k16 with BF16
// operands (weights and activations rounded to BF16 when staged in shared
// memory; FP32 master weights) and FP32 accumulation. The products are small
// (rows = nodes or edges, 128 columns) and latency-bound, which is why they use
// the warp-level MMA rather than tcgen05 tiles with TMEM. Weight gradients
// reduce over rows with a fixed split-K partition and a fixed-order
// reduction, so training steps are deterministic. Aggregations use CSR
// segment sums (edges sorted by destination; a permutation sorted by source).
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/vqemps_mpnn.h"

namespace {

constexpr int GM_BM = 64, GM_BN = 128, GM_BK = 32, GM_PAD = 8, GM_THREADS = 128;

// ---- operand views (element (m, k) of A, (k, n) of B) ----------------------
struct ARow {            // A[m * ld + k]
  const float *p; int ld;
  __device__ float operator()(int m, int k) const { return p[(size_t)m * ld + k]; }
};
struct ACat {            // [P | Q] by columns: k < k1 from P, else from Q
  const float *p; int ldp; const float *q; int ldq; int k1;
  __device__ float operator()(int m, int k) const {
    return k < k1 ? p[(size_t)m * ldp + k] : q[(size_t)m * ldq + (k - k1)];
  }
};
struct AGatherCat {      // [X[idx[m]] | Q[m]]: gathered node rows, then edge features
  const float *x; int ldx; const int32_t *idx; const float *q; int ldq; int k1;
  __device__ float operator()(int m, int k) const {
    return k < k1 ? x[(size_t)idx[m] * ldx + k] : q[(size_t)m * ldq + (k - k1)];
  }
};
struct ATCat {           // transposed [P | Q]: A(m, k) = row k, column m of [P | Q]
  const float *p; int ldp; const float *q; int ldq; int m1;
  __device__ float operator()(int m, int k) const {
    return m < m1 ? p[(size_t)k * ldp + m] : q[(size_t)k * ldq + (m - m1)];
  }
};
struct ATGatherCat {     // transposed [X[idx[k]] | Q[k]]
  const float *x; int ldx; const int32_t *idx; const float *q; int ldq; int m1;
  __device__ float operator()(int m, int k) const {
    return m < m1 ? x[(size_t)idx[k] * ldx + m] : q[(size_t)k * ldq + (m - m1)];
  }
};
struct BRow {            // B[k * ld + n]
  const float *p; int ld;
  __device__ float operator()(int k, int n) const { return p[(size_t)k * ld + n]; }
};
struct BT {              // B(k, n) = P[n * ld + k]  (a transposed weight)
  const float *p; int ld;
  __device__ float operator()(int k, int n) const { return p[(size_t)n * ld + k]; }
};

// ---- epilogues -------------------------------------------------------------
enum : int { EP_STORE = 0, EP_RELU = 1, EP_RESID_RELU = 2, EP_PARTIAL = 3 };

struct Epilogue {
  int kind;
  float *out; int ldo;          // EP_STORE / EP_RELU / EP_RESID_RELU (X out) / EP_PARTIAL (partials)
  const float *bias;            // N or null
  const float *resid; int ldr;  // EP_RESID_RELU: X in
  float *relu_out;              // EP_RESID_RELU: R = relu(acc + bias)
  size_t split_stride;          // EP_PARTIAL: M * N per split
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat16 a = __float2bfloat16_rn(lo), b = __float2bfloat16_rn(hi);
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[M x N] = A[M x K] B[K x N] over the k range of split blockIdx.z. A CTA
// owns a 64 x 128 tile; each of its 4 warps computes 16 rows x 128 columns as
// 16 m16n8 accumulator tiles. Operands are staged as BF16 pairs: As[m][k],
// Bs[n][k] (k contiguous, the .col layout of the B fragment).
template <typename LA, typename LB>
__global__ void __launch_bounds__(GM_THREADS)
gemm_bf16_kernel(int M, int N, int K, int k_per_split, LA A, LB B, Epilogue ep) {
  __shared__ __align__(16) __nv_bfloat16 As[GM_BM][GM_BK + GM_PAD];
  __shared__ __align__(16) __nv_bfloat16 Bs[GM_BN][GM_BK + GM_PAD];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int m0 = blockIdx.x * GM_BM, n0 = blockIdx.y * GM_BN;
  const int k_begin = blockIdx.z * k_per_split;
  const int k_end = min(K, k_begin + k_per_split);
  float acc[16][4];
#pragma unroll
  for (int j = 0; j < 16; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  for (int kb = k_begin; kb < k_end; kb += GM_BK) {
    __syncthreads();
    // A tile: 64 x 32 as 1024 bf16 pairs, 8 per thread
    for (int e = tid; e < GM_BM * GM_BK / 2; e += GM_THREADS) {
      const int r = e / (GM_BK / 2), c = (e % (GM_BK / 2)) * 2;
      const int m = m0 + r, k = kb + c;
      const float v0 = (m < M && k < k_end) ? A(m, k) : 0.f;
      const float v1 = (m < M && k + 1 < k_end) ? A(m, k + 1) : 0.f;
      *reinterpret_cast<uint32_t *>(&As[r][c]) = pack_bf16(v0, v1);
    }
    // B tile: 32 x 128 as 2048 bf16 pairs along k, 16 per thread
    for (int e = tid; e < GM_BN * GM_BK / 2; e += GM_THREADS) {
      const int nn = e % GM_BN, c = (e / GM_BN) * 2;
      const int n = n0 + nn, k = kb + c;
      const float v0 = (n < N && k < k_end) ? B(k, n) : 0.f;
      const float v1 = (n < N && k + 1 < k_end) ? B(k + 1, n) : 0.f;
      *reinterpret_cast<uint32_t *>(&Bs[nn][c]) = pack_bf16(v0, v1);
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < GM_BK; ks += 16) {
      uint32_t a[4];
      const int r = warp * 16 + g;
      a[0] = *reinterpret_cast<const uint32_t *>(&As[r][ks + 2 * t]);
      a[1] = *reinterpret_cast<const uint32_t *>(&As[r + 8][ks + 2 * t]);
      a[2] = *reinterpret_cast<const uint32_t *>(&As[r][ks + 2 * t + 8]);
      a[3] = *reinterpret_cast<const uint32_t *>(&As[r + 8][ks + 2 * t + 8]);
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        uint32_t b[2];
        b[0] = *reinterpret_cast<const uint32_t *>(&Bs[j * 8 + g][ks + 2 * t]);
        b[1] = *reinterpret_cast<const uint32_t *>(&Bs[j * 8 + g][ks + 2 * t + 8]);
        mma_bf16(acc[j], a, b);
      }
    }
  }
  // epilogue: acc[j][0..1] -> row g, cols j*8 + 2t + {0,1}; acc[j][2..3] -> row g + 8
#pragma unroll
  for (int j = 0; j < 16; ++j)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int m = m0 + warp * 16 + g + 8 * h;
      if (m >= M) continue;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int n = n0 + j * 8 + 2 * t + q;
        if (n >= N) continue;
        float v = acc[j][2 * h + q];
        if (ep.kind == EP_PARTIAL) {
          ep.out[(size_t)blockIdx.z * ep.split_stride + (size_t)m * N + n] = v;
          continue;
        }
        if (ep.bias) v += ep.bias[n];
        if (ep.kind == EP_RELU) v = fmaxf(v, 0.f);
        if (ep.kind == EP_RESID_RELU) {
          const float r = fmaxf(v, 0.f);
          ep.relu_out[(size_t)m * N + n] = r;
          v = ep.resid[(size_t)m * ep.ldr + n] + r;
        }
        ep.out[(size_t)m * ep.ldo + n] = v;
      }
    }
}

// out[i] = sum over splits s (in order) of partial[s][i]  (+ accumulate flag)
__global__ void split_reduce_kernel(const float *__restrict__ partial, int splits, size_t count,
                                    float *__restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float s = 0.f;
  for (int z = 0; z < splits; ++z) s += partial[(size_t)z * count + i];
  out[i] = s;
}

// column sums of a rows x cols matrix, fixed order (one thread per column)
__global__ void colsum_kernel(const float *__restrict__ x, int rows, int cols, float *__restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += x[(size_t)r * cols + c];
  out[c] = s;
}

// A[i] = mean over edges e in [off[i], off[i+1]) of M[e]  (edges sorted by destination)
__global__ void segment_mean_kernel(const float *__restrict__ Mv, const int32_t *__restrict__ off, int N, int W,
                                    float *__restrict__ out) {
  const int i = blockIdx.x, c = threadIdx.x;
  if (i >= N || c >= W) return;
  const int b = off[i], e = off[i + 1];
  float s = 0.f;
  for (int k = b; k < e; ++k) s += Mv[(size_t)k * W + c];
  out[(size_t)i * W + c] = e > b ? s / (float)(e - b) : 0.f;
}

// S[i] = sum over edges with source i (perm sorted by source) of V[e]
__global__ void segment_sum_perm_kernel(const float *__restrict__ V, const int32_t *__restrict__ perm,
                                        const int32_t *__restrict__ off, int N, int W, float *__restrict__ out) {
  const int i = blockIdx.x, c = threadIdx.x;
  if (i >= N || c >= W) return;
  float s = 0.f;
  for (int k = off[i]; k < off[i + 1]; ++k) s += V[(size_t)perm[k] * W + c];
  out[(size_t)i * W + c] = s;
}

// dV[e] = dA[dst e] / deg(dst e) masked by M[e] > 0
__global__ void msg_backward_kernel(const float *__restrict__ dA, const int32_t *__restrict__ dst,
                                    const int32_t *__restrict__ off, const float *__restrict__ Mv, int E, int W,
                                    float *__restrict__ dV) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)E * W) return;
  const int e = (int)(i / W), c = (int)(i % W);
  const int d = dst[e];
  const float deg = (float)(off[d + 1] - off[d]);
  dV[i] = Mv[i] > 0.f ? dA[(size_t)d * W + c] / deg : 0.f;
}

// y = x masked by m > 0
__global__ void relu_mask_kernel(const float *__restrict__ x, const float *__restrict__ m, size_t n,
                                 float *__restrict__ y) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = m[i] > 0.f ? x[i] : 0.f;
}

// a += b
__global__ void add_kernel(float *__restrict__ a, const float *__restrict__ b, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] += b[i];
}

// split [N x 2W] rows into a += left half, out = right half
__global__ void split_cols_kernel(const float *__restrict__ g, int N, int W, float *__restrict__ dx_acc,
                                  float *__restrict__ da) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)N * W) return;
  const size_t r = i / W, c = i % W;
  dx_acc[i] += g[r * 2 * W + c];
  da[i] = g[r * 2 * W + W + c];
}

// theta = pi tanh(z)
__global__ void head_kernel(const float *__restrict__ z, size_t n, float *__restrict__ theta) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) theta[i] = 3.14159265358979f * tanhf(z[i]);
}

// dz = dtheta * pi (1 - tanh^2 z), from theta = pi tanh z
__global__ void head_backward_kernel(const float *__restrict__ theta, const float *__restrict__ dtheta, size_t n,
                                     float *__restrict__ dz) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float th = theta[i] * (1.0f / 3.14159265358979f);
  dz[i] = dtheta[i] * 3.14159265358979f * (1.f - th * th);
}

// periodic loss: L = sum_i w_i sum_j (1 - cos(theta_ij - t_ij)) / (out * sum_i w_i);
// dtheta = w_i sin(theta_ij - t_ij) / (out * sum w). One CTA, fixed order.
__global__ void loss_kernel(const float *__restrict__ theta, const float *__restrict__ target,
                            const float *__restrict__ weight, int N, int out_per_node, float *__restrict__ loss,
                            float *__restrict__ dtheta) {
  __shared__ float red[256];
  __shared__ float wsum_s;
  const int tid = threadIdx.x;
  float ws = 0.f;
  for (int i = tid; i < N; i += 256) ws += weight ? weight[i] : 1.f;
  red[tid] = ws;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (tid < s) red[tid] += red[tid + s];
    __syncthreads();
  }
  if (tid == 0) wsum_s = red[0] > 0.f ? red[0] : 1.f;
  __syncthreads();
  const float scale = 1.f / (wsum_s * out_per_node);
  float l = 0.f;
  for (int i = tid; i < N * out_per_node; i += 256) {
    const float w = weight ? weight[i / out_per_node] : 1.f;
    const float d = theta[i] - target[i];
    l += w * (1.f - cosf(d));
    if (dtheta) dtheta[i] = w * sinf(d) * scale;
  }
  __syncthreads();
  red[tid] = l;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (tid < s) red[tid] += red[tid + s];
    __syncthreads();
  }
  if (tid == 0 && loss) *loss = red[0] * scale;
}

__global__ void adam_kernel(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, size_t n, float lr, float b1, float b2, float eps, float wd,
                            float c1, float c2) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] + wd * w[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

template <typename T>
struct Buf {
  T *ptr = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t count) {
    if (count <= cap) return cudaSuccess;
    cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) cap = count;
    return e;
  }
  ~Buf() { cudaFree(ptr); }
};

unsigned grid1(size_t n, int block = 256) { return (unsigned)((n + block - 1) / block); }

}  // namespace

struct vqemps_mpnn {
  int device = 0, node_in = 0, edge_in = 0, width = 0, layers = 0, out = 0;
  std::string err;
  // parameter offsets (floats) in the flat vector
  size_t o_win, o_bin, o_wo, o_bo, count;
  std::vector<size_t> o_wm, o_bm, o_wu, o_bu;
  Buf<float> params, adam_m, adam_v;
  long long adam_t = 0;
  // activations of the last forward
  int N = 0, E = 0;
  Buf<float> X[8], Mv[8], Agg[8], R[8], Z, theta;
  // backward scratch
  Buf<float> dX, dXn, dZ, dU, dA, dV, S, G, partial, tmp;
};

static int fail(vqemps_mpnn *net, int code, const std::string &msg) {
  if (net) net->err = msg;
  return code;
}

#define MPNN_TRY(net, expr)                                                                  \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess)                                                                   \
      return fail(net, VQEMPS_MPNN_CUDA_ERROR, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

template <typename LA, typename LB>
static cudaError_t gemm(int M, int N, int K, LA A, LB B, Epilogue ep, cudaStream_t st, int splits = 1) {
  if (M <= 0 || N <= 0) return cudaSuccess;
  int per = K;
  if (splits > 1) per = ((K + splits - 1) / splits + GM_BK - 1) / GM_BK * GM_BK;
  const int z = per > 0 ? (K + per - 1) / per : 1;
  dim3 grid((M + GM_BM - 1) / GM_BM, (N + GM_BN - 1) / GM_BN, std::max(z, 1));
  gemm_bf16_kernel<LA, LB><<<grid, GM_THREADS, 0, st>>>(M, N, K, std::max(per, 1), A, B, ep);
  return cudaGetLastError();
}

// Weight gradient out[M x N] = A^T-view [M x K] times B [K x N] with a fixed
// split of the K (row) range and an ordered reduction of the partials.
template <typename LA, typename LB>
static int gemm_reduce(vqemps_mpnn *net, int M, int N, int K, LA A, LB B, float *out, cudaStream_t st) {
  const int splits = std::max(1, std::min(64, K / 1024));
  const int per = ((K + splits - 1) / splits + GM_BK - 1) / GM_BK * GM_BK;
  const int z = std::max(1, (K + per - 1) / per);
  MPNN_TRY(net, net->partial.ensure((size_t)z * M * N));
  Epilogue ep{};
  ep.kind = EP_PARTIAL;
  ep.out = net->partial.ptr;
  ep.split_stride = (size_t)M * N;
  dim3 grid((M + GM_BM - 1) / GM_BM, (N + GM_BN - 1) / GM_BN, z);
  gemm_bf16_kernel<LA, LB><<<grid, GM_THREADS, 0, st>>>(M, N, K, per, A, B, ep);
  MPNN_TRY(net, cudaGetLastError());
  split_reduce_kernel<<<grid1((size_t)M * N), 256, 0, st>>>(net->partial.ptr, z, (size_t)M * N, out);
  MPNN_TRY(net, cudaGetLastError());
  return VQEMPS_MPNN_OK;
}

extern "C" int vqemps_mpnn_create(int device, int node_in, int edge_in, int width, int layers, int out_per_node,
                                  vqemps_mpnn **out) {
  if (!out) return VQEMPS_MPNN_INVALID;
  *out = nullptr;
  if (node_in < 1 || edge_in < 0 || width < 16 || width > GM_BN || width % 16 || layers < 0 || layers > 7 ||
      out_per_node < 1)
    return VQEMPS_MPNN_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return VQEMPS_MPNN_CUDA_ERROR;
  auto *net = new vqemps_mpnn();
  net->device = device;
  net->node_in = node_in;
  net->edge_in = edge_in;
  net->width = width;
  net->layers = layers;
  net->out = out_per_node;
  size_t o = 0;
  net->o_win = o; o += (size_t)node_in * width;
  net->o_bin = o; o += width;
  for (int l = 0; l < layers; ++l) {
    net->o_wm.push_back(o); o += (size_t)(width + edge_in) * width;
    net->o_bm.push_back(o); o += width;
    net->o_wu.push_back(o); o += (size_t)2 * width * width;
    net->o_bu.push_back(o); o += width;
  }
  net->o_wo = o; o += (size_t)width * out_per_node;
  net->o_bo = o; o += out_per_node;
  net->count = o;
  if (net->params.ensure(o) != cudaSuccess || net->adam_m.ensure(o) != cudaSuccess ||
      net->adam_v.ensure(o) != cudaSuccess) {
    delete net;
    return VQEMPS_MPNN_CUDA_ERROR;
  }
  cudaMemset(net->params.ptr, 0, o * sizeof(float));
  cudaMemset(net->adam_m.ptr, 0, o * sizeof(float));
  cudaMemset(net->adam_v.ptr, 0, o * sizeof(float));
  *out = net;
  return VQEMPS_MPNN_OK;
}

extern "C" int vqemps_mpnn_destroy(vqemps_mpnn *net) {
  if (!net) return VQEMPS_MPNN_OK;
  cudaSetDevice(net->device);
  delete net;
  return VQEMPS_MPNN_OK;
}

extern "C" const char *vqemps_mpnn_last_error(const vqemps_mpnn *net) {
  return net ? net->err.c_str() : "null network";
}

extern "C" int vqemps_mpnn_num_params(const vqemps_mpnn *net, int64_t *count) {
  if (!net || !count) return VQEMPS_MPNN_INVALID;
  *count = (int64_t)net->count;
  return VQEMPS_MPNN_OK;
}

extern "C" int vqemps_mpnn_set_params(vqemps_mpnn *net, const float *host, int64_t count) {
  if (!net || !host || count != (int64_t)net->count) return fail(net, VQEMPS_MPNN_INVALID, "bad parameter count");
  MPNN_TRY(net, cudaSetDevice(net->device));
  MPNN_TRY(net, cudaMemcpy(net->params.ptr, host, count * sizeof(float), cudaMemcpyHostToDevice));
  MPNN_TRY(net, cudaMemset(net->adam_m.ptr, 0, count * sizeof(float)));
  MPNN_TRY(net, cudaMemset(net->adam_v.ptr, 0, count * sizeof(float)));
  net->adam_t = 0;
  return VQEMPS_MPNN_OK;
}

extern "C" int vqemps_mpnn_get_params(vqemps_mpnn *net, float *host, int64_t count) {
  if (!net || !host || count != (int64_t)net->count) return fail(net, VQEMPS_MPNN_INVALID, "bad parameter count");
  MPNN_TRY(net, cudaSetDevice(net->device));
  MPNN_TRY(net, cudaMemcpy(host, net->params.ptr, count * sizeof(float), cudaMemcpyDeviceToHost));
  return VQEMPS_MPNN_OK;
}

static int check_graph(vqemps_mpnn *net, const vqemps_graph *gr) {
  if (!gr || gr->num_nodes < 1 || gr->num_edges < 0 || !gr->node_feat || !gr->dst_off ||
      (gr->num_edges > 0 && (!gr->edge_src || !gr->edge_dst || !gr->src_perm || !gr->src_off ||
                             (net->edge_in > 0 && !gr->edge_feat))))
    return fail(net, VQEMPS_MPNN_INVALID, "bad graph");
  return VQEMPS_MPNN_OK;
}

extern "C" int vqemps_mpnn_forward(vqemps_mpnn *net, const vqemps_graph *gr, float *angles_dev, void *stream) {
  if (!net) return VQEMPS_MPNN_INVALID;
  int rc = check_graph(net, gr);
  if (rc) return rc;
  MPNN_TRY(net, cudaSetDevice(net->device));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int N = gr->num_nodes, E = gr->num_edges, W = net->width, L = net->layers;
  const float *P = net->params.ptr;
  net->N = N;
  net->E = E;
  for (int l = 0; l <= L; ++l) MPNN_TRY(net, net->X[l].ensure((size_t)N * W));
  for (int l = 0; l < L; ++l) {
    MPNN_TRY(net, net->Mv[l].ensure((size_t)std::max(E, 1) * W));
    MPNN_TRY(net, net->Agg[l].ensure((size_t)N * W));
    MPNN_TRY(net, net->R[l].ensure((size_t)N * W));
  }
  MPNN_TRY(net, net->Z.ensure((size_t)N * net->out));
  MPNN_TRY(net, net->theta.ensure((size_t)N * net->out));
  // encoder
  Epilogue ep{};
  ep.kind = EP_RELU; ep.out = net->X[0].ptr; ep.ldo = W; ep.bias = P + net->o_bin;
  MPNN_TRY(net, gemm(N, W, net->node_in, ARow{gr->node_feat, net->node_in}, BRow{P + net->o_win, W}, ep, st));
  for (int l = 0; l < L; ++l) {
    if (E > 0) {
      Epilogue em{};
      em.kind = EP_RELU; em.out = net->Mv[l].ptr; em.ldo = W; em.bias = P + net->o_bm[l];
      MPNN_TRY(net, gemm(E, W, W + net->edge_in,
                         AGatherCat{net->X[l].ptr, W, gr->edge_src, gr->edge_feat, net->edge_in, W},
                         BRow{P + net->o_wm[l], W}, em, st));
    }
    segment_mean_kernel<<<N, W, 0, st>>>(net->Mv[l].ptr, gr->dst_off, N, W, net->Agg[l].ptr);
    MPNN_TRY(net, cudaGetLastError());
    Epilogue eu{};
    eu.kind = EP_RESID_RELU; eu.out = net->X[l + 1].ptr; eu.ldo = W; eu.bias = P + net->o_bu[l];
    eu.resid = net->X[l].ptr; eu.ldr = W; eu.relu_out = net->R[l].ptr;
    MPNN_TRY(net, gemm(N, W, 2 * W, ACat{net->X[l].ptr, W, net->Agg[l].ptr, W, W}, BRow{P + net->o_wu[l], W}, eu,
                       st));
  }
  Epilogue eo{};
  eo.kind = EP_STORE; eo.out = net->Z.ptr; eo.ldo = net->out; eo.bias = P + net->o_bo;
  MPNN_TRY(net, gemm(N, net->out, W, ARow{net->X[L].ptr, W}, BRow{P + net->o_wo, net->out}, eo, st));
  head_kernel<<<grid1((size_t)N * net->out), 256, 0, st>>>(net->Z.ptr, (size_t)N * net->out, net->theta.ptr);
  MPNN_TRY(net, cudaGetLastError());
  if (angles_dev)
    MPNN_TRY(net, cudaMemcpyAsync(angles_dev, net->theta.ptr, sizeof(float) * N * net->out,
                                  cudaMemcpyDeviceToDevice, st));
  return VQEMPS_MPNN_OK;
}

extern "C" int vqemps_mpnn_loss(vqemps_mpnn *net, const float *target_dev, const float *node_weight_dev,
                                float *loss_dev, float *dangles_dev, void *stream) {
  if (!net || !target_dev || net->N < 1) return fail(net, VQEMPS_MPNN_INVALID, "run forward first");
  MPNN_TRY(net, cudaSetDevice(net->device));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  loss_kernel<<<1, 256, 0, st>>>(net->theta.ptr, target_dev, node_weight_dev, net->N, net->out, loss_dev,
                                 dangles_dev);
  MPNN_TRY(net, cudaGetLastError());
  return VQEMPS_MPNN_OK;
}

extern "C" int vqemps_mpnn_backward(vqemps_mpnn *net, const vqemps_graph *gr, const float *dangles_dev,
                                    float *grad_dev, void *stream) {
  if (!net) return VQEMPS_MPNN_INVALID;
  int rc = check_graph(net, gr);
  if (rc) return rc;
  if (gr->num_nodes != net->N || gr->num_edges != net->E || !dangles_dev || !grad_dev)
    return fail(net, VQEMPS_MPNN_INVALID, "backward needs the forward's graph");
  MPNN_TRY(net, cudaSetDevice(net->device));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const int N = net->N, E = net->E, W = net->width, L = net->layers, O = net->out;
  const float *P = net->params.ptr;
  MPNN_TRY(net, net->dZ.ensure((size_t)N * O));
  MPNN_TRY(net, net->dX.ensure((size_t)N * W));
  MPNN_TRY(net, net->dXn.ensure((size_t)N * W));
  MPNN_TRY(net, net->dU.ensure((size_t)N * W));
  MPNN_TRY(net, net->dA.ensure((size_t)N * W));
  MPNN_TRY(net, net->S.ensure((size_t)N * W));
  MPNN_TRY(net, net->G.ensure((size_t)N * 2 * W));
  MPNN_TRY(net, net->dV.ensure((size_t)std::max(E, 1) * W));
  // head
  head_backward_kernel<<<grid1((size_t)N * O), 256, 0, st>>>(net->theta.ptr, dangles_dev, (size_t)N * O,
                                                             net->dZ.ptr);
  MPNN_TRY(net, cudaGetLastError());
  rc = gemm_reduce(net, W, O, N, ATCat{net->X[L].ptr, W, nullptr, 0, W}, BRow{net->dZ.ptr, O}, grad_dev + net->o_wo,
                   st);
  if (rc) return rc;
  colsum_kernel<<<grid1(O, 128), 128, 0, st>>>(net->dZ.ptr, N, O, grad_dev + net->o_bo);
  Epilogue ex{};
  ex.kind = EP_STORE; ex.out = net->dX.ptr; ex.ldo = W;
  MPNN_TRY(net, gemm(N, W, O, ARow{net->dZ.ptr, O}, BT{P + net->o_wo, O}, ex, st));
  for (int l = L - 1; l >= 0; --l) {
    // update: X_{l+1} = X_l + R_l, R_l = relu([X_l | A_l] Wu + bu)
    relu_mask_kernel<<<grid1((size_t)N * W), 256, 0, st>>>(net->dX.ptr, net->R[l].ptr, (size_t)N * W, net->dU.ptr);
    MPNN_TRY(net, cudaGetLastError());
    rc = gemm_reduce(net, 2 * W, W, N, ATCat{net->X[l].ptr, W, net->Agg[l].ptr, W, W}, BRow{net->dU.ptr, W},
                     grad_dev + net->o_wu[l], st);
    if (rc) return rc;
    colsum_kernel<<<grid1(W, 128), 128, 0, st>>>(net->dU.ptr, N, W, grad_dev + net->o_bu[l]);
    Epilogue eg{};
    eg.kind = EP_STORE; eg.out = net->G.ptr; eg.ldo = 2 * W;
    MPNN_TRY(net, gemm(N, 2 * W, W, ARow{net->dU.ptr, W}, BT{P + net->o_wu[l], W}, eg, st));
    // dX_l = dX_{l+1} (residual) + G[:, :W];  dA = G[:, W:]
    split_cols_kernel<<<grid1((size_t)N * W), 256, 0, st>>>(net->G.ptr, N, W, net->dX.ptr, net->dA.ptr);
    MPNN_TRY(net, cudaGetLastError());
    if (E > 0) {
      msg_backward_kernel<<<grid1((size_t)E * W), 256, 0, st>>>(net->dA.ptr, gr->edge_dst, gr->dst_off,
                                                                 net->Mv[l].ptr, E, W, net->dV.ptr);
      MPNN_TRY(net, cudaGetLastError());
      rc = gemm_reduce(net, W + net->edge_in, W, E,
                       ATGatherCat{net->X[l].ptr, W, gr->edge_src, gr->edge_feat, net->edge_in, W},
                       BRow{net->dV.ptr, W}, grad_dev + net->o_wm[l], st);
      if (rc) return rc;
      colsum_kernel<<<grid1(W, 128), 128, 0, st>>>(net->dV.ptr, E, W, grad_dev + net->o_bm[l]);
      segment_sum_perm_kernel<<<N, W, 0, st>>>(net->dV.ptr, gr->src_perm, gr->src_off, N, W, net->S.ptr);
      MPNN_TRY(net, cudaGetLastError());
      Epilogue es{};
      es.kind = EP_STORE; es.out = net->dXn.ptr; es.ldo = W;
      MPNN_TRY(net, gemm(N, W, W, ARow{net->S.ptr, W}, BT{P + net->o_wm[l], W}, es, st));
      add_kernel<<<grid1((size_t)N * W), 256, 0, st>>>(net->dX.ptr, net->dXn.ptr, (size_t)N * W);
      MPNN_TRY(net, cudaGetLastError());
    } else {
      MPNN_TRY(net, cudaMemsetAsync(grad_dev + net->o_wm[l], 0,
                                    sizeof(float) * ((size_t)(W + net->edge_in) * W + W), st));
    }
  }
  // encoder: X0 = relu(F Win + bin)
  relu_mask_kernel<<<grid1((size_t)N * W), 256, 0, st>>>(net->dX.ptr, net->X[0].ptr, (size_t)N * W, net->dU.ptr);
  MPNN_TRY(net, cudaGetLastError());
  rc = gemm_reduce(net, net->node_in, W, N, ATCat{gr->node_feat, net->node_in, nullptr, 0, net->node_in},
                   BRow{net->dU.ptr, W}, grad_dev + net->o_win, st);
  if (rc) return rc;
  colsum_kernel<<<grid1(W, 128), 128, 0, st>>>(net->dU.ptr, N, W, grad_dev + net->o_bin);
  MPNN_TRY(net, cudaGetLastError());
  return VQEMPS_MPNN_OK;
}

extern "C" int vqemps_mpnn_adam_step(vqemps_mpnn *net, const float *grad_dev, float lr, float beta1, float beta2,
                                     float eps, float weight_decay, void *stream) {
  if (!net || !grad_dev) return VQEMPS_MPNN_INVALID;
  MPNN_TRY(net, cudaSetDevice(net->device));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  net->adam_t += 1;
  const float c1 = 1.f - powf(beta1, (float)net->adam_t);
  const float c2 = 1.f - powf(beta2, (float)net->adam_t);
  adam_kernel<<<grid1(net->count), 256, 0, st>>>(net->params.ptr, grad_dev, net->adam_m.ptr, net->adam_v.ptr,
                                                 net->count, lr, beta1, beta2, eps, weight_decay, c1, c2);
  MPNN_TRY(net, cudaGetLastError());
  return VQEMPS_MPNN_OK;
}
