// Mixed-precision device solve: the RGF sweep in FP32 on the tensor cores,
// the contact self-energies, broadenings and the trace in FP64.
//
// Same contract as rgf_f64_global_kernel (negfpy core/negf.py:72-357): per
// point Sigma = V g V^H for both contacts from the FP64 surface GFs, the
// left-connected sweep g_l = (z - D_l - C^H g_{l-1} C [- Sigma_R])^-1 with
// G_{0,l} = G_{0,l-1} C g_l, and T = Re Tr[Gamma_L G Gamma_R G^H].
//
//   * FP64: z, Sigma_L, Sigma_R (DMMA), Gamma_L, Gamma_R, and the trace
//     (G_{0,L-1} widened to FP64, two DMMA products, FP64 dot product).
//   * FP32: every sweep matrix (g_l, C, W, U, G_0, M) and its inverse.  The
//     products are split 3 x TF32 on mma.sync m16n8k8 (a = a_hi + a_lo with
//     both halves rounded to TF32; a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi,
//     accumulated in FP32), about FP32 accuracy at 12 tensor instructions per
//     complex k-chunk.  The inverse is the blocked division-free Gauss-Jordan
//     of the FP64 kernels in FP32 with the rank-8 update on the same 3 x TF32
//     products.
//
// A point whose FP32 sweep meets a singular or non-finite pivot reports the
// status; the host re-solves those points with the FP64 kernel.
#include "negf_common.cuh"
#include "negf_f64.h"
#include "negf_mixed.cuh"
#include "negf_tiles.cuh"

namespace negf {
namespace mixed {

__global__ void __launch_bounds__(kThreads) rgf_mixed_kernel(RgfArgs a, int NP, unsigned char* ws) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const GJS32 sh = carve32(smraw, NP);
  double* red = reinterpret_cast<double*>(smraw + ((gjs32_bytes(NP) + 15) / 16) * 16);
  __shared__ int s_point;
  const int n = a.n, tid = threadIdx.x;
  unsigned char* blk = ws + (long long)blockIdx.x * mixed_ws_bytes_per_block(NP, n);

  for (;;) {
    if (tid == 0) s_point = (int)atomicAdd(a.counter, 1u);
    __syncthreads();
    const int p = s_point;
    __syncthreads();
    if (p >= a.batch) break;
    const int lst = a.lead_status ? a.lead_status[p] : 0;
    if (lst != kOk) {
      if (tid == 0) {
        a.T_out[p] = __longlong_as_double(0x7ff8000000000000ULL);
        if (a.status_out) a.status_out[p] = lst;
      }
      continue;
    }
    const long long k = a.kidx ? (long long)a.kidx[p] : 0;
    glob::RgfPoint q;
    q.n = n;
    q.nl = a.nl;
    q.nr = a.nr;
    q.L = a.L;
    q.D = a.D + k * a.d_ks;
    q.d_ls = a.d_ls;
    q.C = a.C + k * a.c_ks;
    q.c_ls = a.c_ls;
    q.VL = a.VL + k * a.vl_ks;
    q.VR = a.VR + k * a.vr_ks;
    q.gL = a.gL + (long long)p * a.gl_ps;
    q.gR = a.gR + (long long)p * a.gr_ps;
    q.z = glob::z_of(a.omega[p], a.eta_dev[p]);
    double tval = 0.0;
    const int status = rgf_point_mixed(q, NP, blk, sh, red, &tval);
    if (tid == 0) {
      a.T_out[p] = (status == kOk) ? tval : __longlong_as_double(0x7ff8000000000000ULL);
      if (a.status_out) a.status_out[p] = status;
    }
    __syncthreads();
  }
}

size_t mixed_smem_bytes(int np) { return ((gjs32_bytes(np) + 15) / 16) * 16 + 40 * 8; }

}  // namespace mixed

int mixed_order(int n) {
  if (n <= 0 || n > 256) return 0;
  return (n + 15) / 16 * 16;
}
int rgf_mixed_grid(int np) {
  const size_t sm = mixed::mixed_smem_bytes(np);
  if (cudaFuncSetAttribute(mixed::rgf_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) !=
      cudaSuccess)
    return -3;
  int nb = 0, dev = 0, nsm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mixed::rgf_mixed_kernel, mixed::kThreads, sm) != cudaSuccess ||
      nb <= 0)
    return -3;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nb * nsm;
}
size_t rgf_mixed_ws_bytes(int np, int n, int grid) { return (size_t)grid * mixed::mixed_ws_bytes_per_block(np, n); }
int rgf_mixed_launch(const RgfArgs& a, int np, int grid, void* ws, cudaStream_t st) {
  if (a.batch <= 0) return 0;
  mixed::rgf_mixed_kernel<<<grid, mixed::kThreads, mixed::mixed_smem_bytes(np), st>>>(
      a, np, static_cast<unsigned char*>(ws));
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace negf
