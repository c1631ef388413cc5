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
#include <atomic>
#include <cstdlib>

#include "negf_common.cuh"
#include "negf_f64.h"
#include "negf_mixed.cuh"
#include "negf_tiles.cuh"

namespace negf {
namespace mixed {

// Dynamic shared memory: [tcgen05 stage and mbarrier (TC only) | GJ panel,
// pivot bookkeeping | reduction scratch].  With TC at least 80 KB, so that at
// most two blocks share an SM and their TMEM (2 x 256 columns) always fits.
__host__ __device__ inline size_t tc_bytes(int np) { return ((tc::stage_bytes(np) + 16 + 127) / 128) * 128; }
template <bool TC>
size_t mixed_smem(int np) {
  const size_t base = ((gjs32_bytes(np) + 15) / 16) * 16 + 40 * 8;
  if (!TC) return base;
  const size_t need = tc_bytes(np) + base;
  return need > 80 * 1024 ? need : 80 * 1024;
}

template <bool TC>
__global__ void __launch_bounds__(kThreads, 2) rgf_mixed_kernel(RgfArgs a, int NP, unsigned char* ws) {
  extern __shared__ __align__(128) unsigned char smraw[];
  unsigned char* gj = smraw + (TC ? tc_bytes(NP) : 0);
  const GJS32 sh = carve32(gj, NP);
  double* red = reinterpret_cast<double*>(gj + ((gjs32_bytes(NP) + 15) / 16) * 16);
  __shared__ int s_point;
  __shared__ uint32_t s_tmem;
  __shared__ int s_tcerr;
  const int n = a.n, tid = threadIdx.x;
  unsigned char* blk = ws + (long long)blockIdx.x * mixed_ws_bytes_per_block(NP, n);
  tc::Ctx tcx;
  if constexpr (TC) tcx = tc::setup(smraw, NP, &s_tmem, &s_tcerr);

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
    const int status = rgf_point_mixed<TC>(q, NP, blk, sh, red, &tval, &tcx);
    if (tid == 0) {
      a.T_out[p] = (status == kOk) ? tval : __longlong_as_double(0x7ff8000000000000ULL);
      if (a.status_out) a.status_out[p] = status;
    }
    __syncthreads();
  }
  if constexpr (TC) tc::teardown(tcx);
}

}  // namespace mixed

// Product tiling of the FP32 sweeps per padded order (index np / 16):
// -1 the default, 0 mma.sync 16 x 16 warp tiles, 1 tcgen05 128 x NP tiles
// (orders up to 128).  Set by negf_set_fp32_product_path (the autotuner);
// the default is mma.sync, or NEGF_TC=1 / 0 in the environment.
std::atomic<int> g_fp32_path[17] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
namespace mixed {
bool use_tc(int np) {
  if (np > tc::kMaxNP || np <= 0) return false;
  const int v = g_fp32_path[np / 16].load();
  if (v >= 0) return v == 1;
  static const int env = [] {
    const char* e = getenv("NEGF_TC");
    return (e && e[0] == '1') ? 1 : 0;
  }();
  return env == 1;
}
}  // namespace mixed
int set_fp32_product_path(int np, int path) {
  if (np <= 0 || np > 256 || np % 16 != 0) return -1;
  if (path == 1 && np > tc::kMaxNP) return -2;
  g_fp32_path[np / 16].store(path < 0 ? -1 : path);
  return mixed::use_tc(np) ? 1 : 0;
}
int mixed_order(int n) {
  if (n <= 0 || n > 256) return 0;
  return (n + 15) / 16 * 16;
}
int rgf_mixed_grid(int np) {
  const bool tcp = mixed::use_tc(np);
  const size_t sm = tcp ? mixed::mixed_smem<true>(np) : mixed::mixed_smem<false>(np);
  auto kernel = tcp ? mixed::rgf_mixed_kernel<true> : mixed::rgf_mixed_kernel<false>;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return -3;
  int nb = 0, dev = 0, nsm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, mixed::kThreads, sm) != cudaSuccess || nb <= 0)
    return -3;
  if (tcp && nb > 2) nb = 2;  // two blocks' TMEM per SM
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nb * nsm;
}
size_t rgf_mixed_ws_bytes(int np, int n, int grid) { return (size_t)grid * mixed::mixed_ws_bytes_per_block(np, n); }
int rgf_mixed_launch(const RgfArgs& a, int np, int grid, void* ws, cudaStream_t st) {
  if (a.batch <= 0) return 0;
  if (mixed::use_tc(np)) {
    mixed::rgf_mixed_kernel<true><<<grid, mixed::kThreads, mixed::mixed_smem<true>(np), st>>>(
        a, np, static_cast<unsigned char*>(ws));
  } else {
    mixed::rgf_mixed_kernel<false><<<grid, mixed::kThreads, mixed::mixed_smem<false>(np), st>>>(
        a, np, static_cast<unsigned char*>(ws));
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace negf
