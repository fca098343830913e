// Shared device helpers: FP64 complex arithmetic on double2 and engine constants.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace vqemps {

// Padded bond dimension of every site tensor in HBM. A site tensor is
// [CHI][2][CHI] complex doubles = 8 KiB; bonds smaller than CHI are zero padded.
constexpr int CHI = 16;
constexpr int SITE_ELEMS = CHI * 2 * CHI;     // 512 complex
constexpr int ENV_ELEMS = CHI * CHI;          // 256 complex (4 KiB)

typedef double2 cplx;

__host__ __device__ __forceinline__ cplx cmake(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cconj(cplx a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return make_double2(a.x * s, a.y * s); }
// acc += a * b
__device__ __forceinline__ void cfma(cplx &acc, cplx a, cplx b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
__device__ __forceinline__ void cfma_conj(cplx &acc, cplx a, cplx b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
__device__ __forceinline__ double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }

// Status words written by kernels (mirrors vqemps_status).
enum : int32_t { ST_OK = 0, ST_INSUFFICIENT = 1, ST_NONFINITE = 2, ST_INVALID = 3, ST_TIMEOUT = 5 };

}  // namespace vqemps
