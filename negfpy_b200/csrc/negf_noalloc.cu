// Allocation-free variant of the batched device solve (negf_rgf_transmission_f64).
//
// Some callers cannot allocate device memory at the moment they call the
// library: a host program that sized all of its GPU memory up front (a
// workflow driver or service with a fixed HBM budget and its own pool), or
// code bound through the C ABI from a language with no CUDA allocator at
// hand.  For them this entry point takes the same inputs and outputs as the
// allocating one but needs no workspace: its scratch (the work counter and
// the per-block self-energy buffers) lives in one static device array,
// g_noalloc_scratch, of kNoAllocScratchBytes = 16 MiB, which every GPU that
// loads the library keeps until the process exits.
//
// The array's host-side name is only a stand-in for the device copy, so the
// device address is looked up with cudaGetSymbolAddress once per device, the
// first time the entry point runs on that device (with it current), and
// cached.  Because that first call does this set-up, make it before any
// stream capture.  All calls share the array and it keeps the last call's
// contents; the work counter is cleared on the caller's stream at the start
// of every call.  Calls whose GPU work overlaps (different streams, or
// different host threads on the same device) race on the array and must not
// be issued concurrently.
#include <cstdio>
#include <mutex>

#include "../../include/negf_b200.h"
#include "negf_f64.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr size_t kCounterBytes = 256;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Failures go through the library's shared per-thread message, so
// negf_last_error() describes them like those of every other entry point.
int noalloc_fail(int code, const char* msg) { return negf::record_error(code, msg); }

// Device address of the scratch array on the current device (looked up once).
void* scratch_address(int* rc) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    *rc = noalloc_fail(NEGF_ECUDA, "negf_rgf_transmission_f64_noalloc: no current CUDA device");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_scratch_addr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      char msg[256];
      snprintf(msg, sizeof(msg), "negf_rgf_transmission_f64_noalloc: cudaGetSymbolAddress: %s",
               cudaGetErrorString(e));
      *rc = noalloc_fail(NEGF_ECUDA, msg);
      return nullptr;
    }
    g_scratch_addr[dev] = p;
  }
  *rc = 0;
  return g_scratch_addr[dev];
}

int max3i(int a, int b, int c) { return a > b ? (a > c ? a : c) : (b > c ? b : c); }

}  // namespace

extern "C" {

int negf_rgf_transmission_f64_noalloc(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch,
                                      const double* onsite, long long onsite_kstride, long long onsite_lstride,
                                      const double* coupling, long long coupling_kstride,
                                      long long coupling_lstride, const double* v_left, long long v_left_kstride,
                                      const double* v_right, long long v_right_kstride, const double* g_left,
                                      long long g_left_pstride, const double* g_right, long long g_right_pstride,
                                      const int* k_index, const double* omega, const double* eta_device,
                                      const int* lead_status, double* t_out, int* status_out, void* stream) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0 || n_layers <= 0 || batch < 0)
    return noalloc_fail(NEGF_EINVAL, "negf_rgf_transmission_f64_noalloc: sizes must be positive");
  if (!onsite || !v_left || !v_right || !g_left || !g_right || !omega || !eta_device || !t_out)
    return noalloc_fail(NEGF_EINVAL, "negf_rgf_transmission_f64_noalloc: null pointer");
  if (n_layers > 1 && !coupling) return noalloc_fail(NEGF_EINVAL, "negf_rgf_transmission_f64_noalloc: null coupling");
  if (onsite_kstride < 0 || onsite_lstride < 0 || coupling_kstride < 0 || coupling_lstride < 0 ||
      v_left_kstride < 0 || v_right_kstride < 0 || g_left_pstride < 0 || g_right_pstride < 0)
    return noalloc_fail(NEGF_EINVAL, "negf_rgf_transmission_f64_noalloc: negative stride");
  const int np = negf::padded_order(max3i(n_dev, n_lead_l, n_lead_r));
  if (np == 0)
    return noalloc_fail(NEGF_EUNSUPPORTED, "negf_rgf_transmission_f64_noalloc: block order above 48 is not supported");
  // Scratch per persistent block: two n_dev x n_dev complex self-energies,
  // at most 72 KiB for n_dev <= 48, so at least 227 blocks fit the array.
  const size_t per_block = size_t(2) * n_dev * n_dev * 16;
  int rc = 0;
  void* base = scratch_address(&rc);
  if (!base) return rc;
  if (batch == 0) return 0;
  int grid = 0;
  if (np != 1) {
    grid = negf::rgf_f64_grid(np);
    if (grid <= 0) return noalloc_fail(NEGF_ECUDA, "negf_rgf_transmission_f64_noalloc: occupancy query failed");
    // The kernel takes work from a counter, so any grid >= 1 is valid.  On a
    // 148-SM B200 the occupancy grid stays below the fit: registers and
    // shared memory allow 1 block per SM at padded order 48, 2 at 32 and at
    // most 8 at 16 (148, 296 and 1184 blocks), against a fit of at least
    // 227, 511 and 2047 blocks.  The cap only acts on GPUs with more SMs.
    const size_t fit = (kNoAllocScratchBytes - kCounterBytes) / per_block;
    if ((size_t)grid > fit) grid = (int)fit;
  }
  negf::RgfArgs a;
  a.n = n_dev;
  a.nl = n_lead_l;
  a.nr = n_lead_r;
  a.L = n_layers;
  a.batch = batch;
  a.D = reinterpret_cast<const double2*>(onsite);
  a.d_ks = onsite_kstride;
  a.d_ls = onsite_lstride;
  a.C = reinterpret_cast<const double2*>(coupling ? coupling : onsite);
  a.c_ks = coupling_kstride;
  a.c_ls = coupling_lstride;
  a.VL = reinterpret_cast<const double2*>(v_left);
  a.vl_ks = v_left_kstride;
  a.VR = reinterpret_cast<const double2*>(v_right);
  a.vr_ks = v_right_kstride;
  a.gL = reinterpret_cast<const double2*>(g_left);
  a.gl_ps = g_left_pstride;
  a.gR = reinterpret_cast<const double2*>(g_right);
  a.gr_ps = g_right_pstride;
  a.kidx = k_index;
  a.omega = omega;
  a.eta_dev = eta_device;
  a.lead_status = lead_status;
  a.T_out = t_out;
  a.status_out = status_out;
  a.counter = reinterpret_cast<unsigned int*>(base);
  a.sigma_ws = reinterpret_cast<double2*>(static_cast<char*>(base) + kCounterBytes);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (np != 1 && cudaMemsetAsync(base, 0, sizeof(unsigned int), st) != cudaSuccess)
    return noalloc_fail(NEGF_ECUDA, "negf_rgf_transmission_f64_noalloc: counter reset failed");
  const int lrc = negf::rgf_f64_launch(a, np, grid, st);
  if (lrc == -2) return noalloc_fail(NEGF_EUNSUPPORTED, "negf_rgf_transmission_f64_noalloc: block order not built");
  if (lrc != 0) return noalloc_fail(NEGF_ECUDA, negf::last_launch_error());
  return 0;
}

}  // extern "C"
