// Batched complex FP32 products on tcgen05 (negf_tcprod.cuh): C_p = op(A_p) op(B_p)
// for P independent n x n matrices, one thread block per product.  The
// building block of the tensor-core device sweeps, exposed on its own so that
// it can be checked against an FP32 reference.
#include "negf_common.cuh"
#include "negf_f64.h"
#include "negf_tcprod.cuh"

namespace negf {
namespace tc {

// Dynamic shared memory of a product block: at least 80 KB, so that at most
// two blocks share an SM and their TMEM (2 x 256 columns) always fits.
__host__ __device__ constexpr size_t block_smem(int np) {
  return stage_bytes(np) + 16 > 80 * 1024 ? stage_bytes(np) + 16 : 80 * 1024;
}

template <bool AC, bool BC>
__global__ void __launch_bounds__(kThreads, 1) cgemm_kernel(int NP, const float2* A, const float2* B, float2* C,
                                                            int* status) {
  extern __shared__ __align__(128) unsigned char smraw[];
  __shared__ uint32_t tslot;
  __shared__ int err;
  Ctx ctx = setup(smraw, NP, &tslot, &err);
  const long long off = (long long)blockIdx.x * NP * NP;
  const bool ok = cprod<AC, BC>(C + off, A + off, B + off, NP, ctx);
  if (threadIdx.x == 0 && status) status[blockIdx.x] = ok ? kOk : kNonFinite;
  teardown(ctx);
}

}  // namespace tc

int tc_cgemm_launch(int np, int batch, const float2* a, const float2* b, float2* c, int conj_a, int conj_b,
                    int* status, cudaStream_t st) {
  if (batch <= 0) return 0;
  const size_t sm = tc::block_smem(np);
  auto launch = [&](auto kernel) {
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return -3;
    kernel<<<batch, tc::kThreads, sm, st>>>(np, a, b, c, status);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
  };
  if (conj_a && conj_b) return launch(tc::cgemm_kernel<true, true>);
  if (conj_a) return launch(tc::cgemm_kernel<true, false>);
  if (conj_b) return launch(tc::cgemm_kernel<false, true>);
  return launch(tc::cgemm_kernel<false, false>);
}

}  // namespace negf
