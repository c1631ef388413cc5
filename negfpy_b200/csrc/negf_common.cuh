// Device helpers shared by the NEGF kernels: complex arithmetic on
// interleaved (re, im) pairs, block reductions, and the per-point status codes.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace negf {

// Per-point numerical status (also the values of the C-ABI status arrays).
enum Status : int {
  kOk = 0,
  kMaxIter = 1,     // Sancho-Rubio did not reach tol within maxiter
  kNonFinite = 2,   // inf/nan appeared
  kSingular = 3,    // exact zero pivot in an inversion
  kRefineFail = 4,  // mixed-precision refinement did not converge
  kBadItem = 5,     // batch item with an out-of-range system, k index or block order
  kUnstable = 6,    // Sancho-Rubio: inf/nan arose inside an iteration from finite blocks
};

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// acc += a * b, four FP64 FMAs.
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// 1 / (a + ib) by Smith's algorithm (R. L. Smith, CACM 5(8), 1962), which
// scales by the larger component to avoid overflow in a^2 + b^2.
__device__ __forceinline__ double2 crecip(double2 v) {
  double a = v.x, b = v.y;
  if (fabs(a) >= fabs(b)) {
    double r = b / a;
    double d = a + b * r;
    return make_double2(1.0 / d, -r / d);
  } else {
    double r = a / b;
    double d = a * r + b;
    return make_double2(r / d, -1.0 / d);
  }
}
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ bool cfinite(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// FP32 -> TF32 with round-to-nearest (ties away), as a bit pattern.
__device__ __forceinline__ unsigned tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
// x = hi + lo with both parts representable in TF32.
__device__ __forceinline__ void split_tf32(float x, unsigned& hi, unsigned& lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - __uint_as_float(hi));
}

// Single precision counterparts for the mixed-precision kernels.
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}

// Block-wide reductions.  `red` must hold at least 33 doubles of shared
// memory; every thread of the block must call with uniform control flow.
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();  // protects `red` from a previous reduction still being read
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double w = lane < nw ? red[lane] : -1.0;
    w = warp_max(w);
    if (lane == 0) red[32] = w;
  }
  __syncthreads();
  return red[32];
}
__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double w = lane < nw ? red[lane] : 0.0;
    w = warp_sum(w);
    if (lane == 0) red[32] = w;
  }
  __syncthreads();
  return red[32];
}
// Returns nonzero in every thread if any thread passed nonzero.
__device__ __forceinline__ int block_any(int v) { return __syncthreads_or(v); }

// The status of a decimation whose products or sums of iteration `it` came
// out non-finite.  negfpy runs each iteration under numpy's floating-point
// traps (core/surface_gf.py:40-56): an overflow or invalid operation in the
// products is "numerically unstable", while inf/nan that came in with the
// blocks pass through quietly and are "non-finite values".  Every iteration
// after the first starts from finite blocks, so only the first can be the
// quiet case.  (An inversion that meets inf/nan stays kNonFinite: numpy's
// inverse runs with the traps off and hands NaN on quietly.)  Every thread
// of the block calls this.
__device__ __forceinline__ int sr_failure_status(int it, int n, const double2* h00, const double2* h01,
                                                 const double2* h10, double2 z) {
  int bad = 0;
  if (it == 1) {
    bad = !(isfinite(z.x) && isfinite(z.y));
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const double2 a = h00[e], b = h01[e], c = h10 ? h10[e] : make_double2(0.0, 0.0);
      bad |= !(isfinite(a.x) && isfinite(a.y) && isfinite(b.x) && isfinite(b.y) && isfinite(c.x) && isfinite(c.y));
    }
  }
  return block_any(bad) ? kNonFinite : kUnstable;
}

}  // namespace negf
