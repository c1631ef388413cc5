// Uneven batch: many independent lead/device/lead systems of different block
// orders, layer counts and k grids in ONE persistent launch.
//
// A work item is (system, k index, omega).  Each block takes items from an
// atomic counter in the order the host gave them (largest estimated cost
// first, so the tail of the launch is short), and runs for its item:
//   1. the left lead's Sancho-Rubio decimation at the lead's own padded order
//      (negfpy core/surface_gf.py:18-81), and the right lead's unless the
//      system's leads are the same,
//   2. the device solve at the system's padded order, in FP64
//      (rgf_point_f64) or with the FP32 sweep (rgf_point_mixed),
// writing T, the status and the decimation sweeps of the item.  Block orders
// up to 256; the per-block workspace and the shared memory are sized for the
// largest order in the batch.
#include <atomic>

#include "../../include/negf_b200.h"
#include "negf_common.cuh"
#include "negf_f64.h"
#include "negf_mixed.cuh"
#include "negf_point.cuh"
#include "negf_tiles.cuh"

namespace negf {
namespace batch {

using glob::kThreads;

struct BatchArgs {
  const NegfBatchSystem* sys;
  int n_systems;
  const int* item_system;
  const int* item_k;
  const double* item_omega;
  int n_items;
  double tol;
  int maxiter;
  double* T_out;
  int* status_out;
  int* iters_out;
  unsigned* counter;
};

__host__ __device__ inline int pad16(int n) { return (n + 15) / 16 * 16; }
// Per-block workspace, in complex128 elements, for padded order NP: the two
// compact lead surface GFs and the scratch of the larger of the decimation
// (7 NP^2), the FP64 device solve (6 NP^2 + 2 n^2) and the mixed one
// (7 NP^2 + 2 n^2 in complex128 units).
__host__ __device__ inline size_t block_elems(int np) { return 2 * (size_t)np * np + 9 * (size_t)np * np; }

// MINB: blocks per SM the register allocation is capped for (1: no cap,
// 2: at most 128 registers a thread, with some spilling).
template <bool MIXED, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) batch_kernel(BatchArgs a, int NPmax, double2* ws) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double* red = reinterpret_cast<double*>(smraw + ((glob::gjs_bytes(NPmax) + 15) / 16) * 16);
  __shared__ int s_item;
  const int tid = threadIdx.x;
  const long long M2max = (long long)NPmax * NPmax;
  double2* base = ws + (long long)blockIdx.x * block_elems(NPmax);
  double2* gl = base;
  double2* gr = base + M2max;
  double2* scratch = base + 2 * M2max;

  for (;;) {
    if (tid == 0) s_item = (int)atomicAdd(a.counter, 1u);
    __syncthreads();
    const int p = s_item;
    __syncthreads();
    if (p >= a.n_items) break;
    const int si = a.item_system[p];
    if (si < 0 || si >= a.n_systems) {
      if (tid == 0) {
        a.T_out[p] = __longlong_as_double(0x7ff8000000000000ULL);
        if (a.status_out) a.status_out[p] = kBadItem;
        if (a.iters_out) a.iters_out[p] = 0;
      }
      continue;
    }
    const NegfBatchSystem& d = a.sys[si];
    const long long k = a.item_k[p];
    const double w = a.item_omega[p];
    const int n = d.n_dev, nl = d.n_lead_l, nr = d.n_lead_r;
    int status = kOk, iters = 0;
    if (k < 0 || k >= d.n_k || n <= 0 || nl <= 0 || nr <= 0 || d.n_layers <= 0 || n > NPmax || nl > NPmax ||
        nr > NPmax || (d.same_leads && nl != nr))
      status = kBadItem;
    // 1. lead surface GFs (compact, row stride = lead order)
    for (int side = 0; side < 2 && status == kOk; ++side) {
      if (side == 1 && d.same_leads) break;
      const int m = side ? nr : nl;
      const int NPl = pad16(m);
      const glob::GJS sh = glob::carve(smraw, NPl);
      const long long ks = side ? d.lead_r_kstride : d.lead_l_kstride;
      const double2* h00 = reinterpret_cast<const double2*>(side ? d.lead_r_h00 : d.lead_l_h00) + k * ks;
      const double2* h01 = reinterpret_cast<const double2*>(side ? d.lead_r_h01 : d.lead_l_h01) + k * ks;
      const double* h10r = side ? d.lead_r_h10 : d.lead_l_h10;
      const double2* h10 = h10r ? reinterpret_cast<const double2*>(h10r) + k * ks : nullptr;
      int it = 0;
      double2* pg = nullptr;
      status = glob::sr_point(m, NPl, h00, h01, h10, glob::z_of(w, d.eta), a.tol, a.maxiter, scratch, sh, red,
                              &it, &pg);
      if (side == 0) iters = it;
      if (status == kOk) {
        double2* dst = side ? gr : gl;
        for (int e = tid; e < m * m; e += kThreads) {
          const int r = e / m, c = e - r * m;
          dst[e] = pg[(long long)r * NPl + c];
        }
      }
      __syncthreads();
    }
    // 2. device solve
    double tval = 0.0;
    if (status == kOk) {
      const int NP = pad16(max(n, max(nl, nr)));
      glob::RgfPoint q;
      q.n = n;
      q.nl = nl;
      q.nr = nr;
      q.L = d.n_layers;
      q.D = reinterpret_cast<const double2*>(d.onsite) + k * d.onsite_kstride;
      q.d_ls = d.onsite_lstride;
      q.C = reinterpret_cast<const double2*>(d.coupling ? d.coupling : d.onsite) + k * d.coupling_kstride;
      q.c_ls = d.coupling_lstride;
      q.VL = reinterpret_cast<const double2*>(d.v_left) + k * d.v_left_kstride;
      q.VR = reinterpret_cast<const double2*>(d.v_right) + k * d.v_right_kstride;
      q.gL = gl;
      q.gR = d.same_leads ? gl : gr;
      q.z = glob::z_of(w, d.eta_device);
      if (MIXED) {
        const mixed::GJS32 sh = mixed::carve32(smraw, NP);
        status = mixed::rgf_point_mixed(q, NP, reinterpret_cast<unsigned char*>(scratch), sh, red, &tval);
      } else {
        const glob::GJS sh = glob::carve(smraw, NP);
        status = glob::rgf_point_f64(q, NP, scratch, sh, red, &tval);
      }
    }
    if (tid == 0) {
      a.T_out[p] = (status == kOk) ? tval : __longlong_as_double(0x7ff8000000000000ULL);
      if (a.status_out) a.status_out[p] = status;
      if (a.iters_out) a.iters_out[p] = iters;
    }
    __syncthreads();
  }
}

size_t smem_bytes(int npmax) { return ((glob::gjs_bytes(npmax) + 15) / 16) * 16 + 40 * 8; }

// Largest dynamic shared memory already configured per (device, variant):
// the attribute is set once, outside any stream capture that replays the launch.
std::atomic<int> g_smem_set[4][64];

template <bool MIXED, int MINB>
int configure(int npmax) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -3;
  const int sm = (int)smem_bytes(npmax);
  std::atomic<int>& cur = g_smem_set[(MIXED ? 2 : 0) + (MINB - 1)][dev];
  if (cur.load() >= sm) return 0;
  if (cudaFuncSetAttribute(batch_kernel<MIXED, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) !=
      cudaSuccess)
    return -3;
  cur.store(sm);
  return 0;
}

template <bool MIXED, int MINB>
int max_grid(int npmax) {
  if (configure<MIXED, MINB>(npmax) != 0) return -3;
  int nb = 0, dev = 0, nsm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch_kernel<MIXED, MINB>, kThreads, smem_bytes(npmax)) !=
          cudaSuccess ||
      nb <= 0)
    return -3;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nb * nsm;
}

template <bool MIXED, int MINB>
int launch_variant(const BatchArgs& a, int npmax, int grid, double2* ws, cudaStream_t st) {
  if (configure<MIXED, MINB>(npmax) != 0) return -3;
  batch_kernel<MIXED, MINB><<<grid, kThreads, smem_bytes(npmax), st>>>(a, npmax, ws);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace batch

int batch_max_grid(int npmax, int mixed, int minb) {
  if (minb == 2) return mixed ? batch::max_grid<true, 2>(npmax) : batch::max_grid<false, 2>(npmax);
  return mixed ? batch::max_grid<true, 1>(npmax) : batch::max_grid<false, 1>(npmax);
}
size_t batch_ws_bytes(int npmax, int grid) { return (size_t)grid * batch::block_elems(npmax) * 16; }
int batch_launch(const NegfBatchSystem* sys, int n_systems, const int* item_system, const int* item_k, const double* item_omega,
                 int n_items, double tol, int maxiter, double* t_out, int* status_out, int* iters_out, int npmax,
                 int mixed, int minb, int grid, void* counter, void* ws, cudaStream_t st) {
  batch::BatchArgs a;
  a.sys = sys;
  a.n_systems = n_systems;
  a.item_system = item_system;
  a.item_k = item_k;
  a.item_omega = item_omega;
  a.n_items = n_items;
  a.tol = tol;
  a.maxiter = maxiter;
  a.T_out = t_out;
  a.status_out = status_out;
  a.iters_out = iters_out;
  a.counter = static_cast<unsigned*>(counter);
  double2* w = static_cast<double2*>(ws);
  if (minb == 2)
    return mixed ? batch::launch_variant<true, 2>(a, npmax, grid, w, st)
                 : batch::launch_variant<false, 2>(a, npmax, grid, w, st);
  return mixed ? batch::launch_variant<true, 1>(a, npmax, grid, w, st)
               : batch::launch_variant<false, 1>(a, npmax, grid, w, st);
}

}  // namespace negf
