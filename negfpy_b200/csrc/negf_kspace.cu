// k-space blocks of a force-constant model for many k at once (negfpy
// models/material_kspace.py:99-128, _sum_k_terms and _build_dynamical_blocks):
//   out[k][i][j] = wr[i] (sum_t Phi_t[i][j] exp(i (ky dy_t + kz dz_t)) + pin delta_ij) wc[j]
// with real terms Phi_t (order N), row / column weights wr, wc (inverse
// square roots of the masses) and an onsite pinning.  One block per
// (k, 256-element tile); the T phases of the block's k are formed once in
// shared memory.  Memory-bound: each term element is read once per k from L2.
#include "../../include/negf_b200.h"
#include "negf_common.cuh"

namespace negf {
namespace {

constexpr int kMaxTerms = 256;

__global__ void phase_sum_kernel(const double* __restrict__ terms, const double* __restrict__ shifts, int T,
                                 const double* __restrict__ kpts, int N, const double* __restrict__ wr,
                                 const double* __restrict__ wc, double pin, double2* __restrict__ out) {
  __shared__ double2 ph[kMaxTerms];
  const int k = blockIdx.y;
  const double ky = kpts[2 * k], kz = kpts[2 * k + 1];
  for (int t = threadIdx.x; t < T; t += blockDim.x) {
    double s, c;
    sincos(ky * shifts[2 * t] + kz * shifts[2 * t + 1], &s, &c);
    ph[t] = make_double2(c, s);
  }
  __syncthreads();
  const long long NN = (long long)N * N;
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= NN) return;
  const int i = (int)(e / N), j = (int)(e - (long long)i * N);
  double re = (i == j) ? pin : 0.0, im = 0.0;
  for (int t = 0; t < T; ++t) {
    const double v = terms[(long long)t * NN + e];
    re = fma(v, ph[t].x, re);
    im = fma(v, ph[t].y, im);
  }
  const double w = wr[i] * wc[j];
  out[(long long)k * NN + e] = make_double2(re * w, im * w);
}

}  // namespace
}  // namespace negf

extern "C" int negf_kspace_blocks_f64(const double* terms, const double* shifts, int n_terms, const double* kpoints,
                                      int n_k, int n, const double* row_weight, const double* col_weight,
                                      double pinning, double* out, void* stream) {
  if (n_terms <= 0 || n_terms > negf::kMaxTerms || n_k < 0 || n <= 0 || !terms || !shifts || !kpoints ||
      !row_weight || !col_weight || !out)
    return NEGF_EINVAL;
  if (n_k == 0) return 0;
  const long long nn = (long long)n * n;
  const dim3 grid((unsigned)((nn + 255) / 256), (unsigned)n_k);
  negf::phase_sum_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      terms, shifts, n_terms, kpoints, n, row_weight, col_weight, pinning, reinterpret_cast<double2*>(out));
  return cudaGetLastError() == cudaSuccess ? 0 : NEGF_ECUDA;
}
