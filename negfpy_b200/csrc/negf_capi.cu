// extern "C" entry points of libnegfb200.so (declared in include/negf_b200.h).
// Argument checks happen here, on the host; the kernels assume valid input.
#include <cstdio>
#include <cstring>

#include "../../include/negf_b200.h"
#include "negf_f64.h"

namespace {
thread_local char g_err[256] = "";

int fail(int code, const char* msg) {
  std::snprintf(g_err, sizeof(g_err), "%s", msg);
  return code;
}
int cuda_fail(const char* where) {
  cudaError_t e = cudaGetLastError();
  std::snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
  return NEGF_ECUDA;
}
inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
constexpr size_t kCounterBytes = 256;
}  // namespace

namespace negf {
int record_error(int code, const char* msg) { return fail(code, msg); }
}  // namespace negf

extern "C" {

int negf_get_version(void) { return NEGF_B200_ABI_VERSION; }

const char* negf_last_error(void) { return g_err; }

int negf_max_order_f64(void) { return 256; }

size_t negf_sgf_workspace_bytes(int n) {
  if (n <= 0 || n > 256) return 0;
  if (n <= 48) return kCounterBytes;
  const int np = negf::global_order(n);
  const int grid = negf::sr_global_grid(np);
  if (grid <= 0) return 0;
  return kCounterBytes + negf::sr_global_ws_bytes(np, grid);
}

int negf_sgf_sr_f64(int n, int batch, const double* h00, const double* h01, const double* h10, long long lead_stride,
                    const int* k_index, const double* omega, const double* eta, double tol, int maxiter,
                    double* g_out, double* dos_out, int* iters_out, int* status_out, void* workspace,
                    size_t workspace_bytes, void* stream) {
  if (n <= 0 || batch < 0) return fail(NEGF_EINVAL, "negf_sgf_sr_f64: n must be positive and batch non-negative");
  if (!h00 || !h01 || !omega || !eta) return fail(NEGF_EINVAL, "negf_sgf_sr_f64: null input pointer");
  if (maxiter <= 0 || !(tol > 0.0)) return fail(NEGF_EINVAL, "negf_sgf_sr_f64: maxiter and tol must be positive");
  if (lead_stride < 0) return fail(NEGF_EINVAL, "negf_sgf_sr_f64: negative lead_stride");
  if (n > 256) return fail(NEGF_EUNSUPPORTED, "negf_sgf_sr_f64: block order above 256");
  negf::SrArgs a;
  a.n = n;
  a.batch = batch;
  a.h00 = reinterpret_cast<const double2*>(h00);
  a.h01 = reinterpret_cast<const double2*>(h01);
  a.h10 = reinterpret_cast<const double2*>(h10);
  a.lead_stride = lead_stride;
  a.kidx = k_index;
  a.omega = omega;
  a.eta = eta;
  a.tol = tol;
  a.maxiter = maxiter;
  a.g_out = reinterpret_cast<double2*>(g_out);
  a.dos_out = dos_out;
  a.iters_out = iters_out;
  a.status_out = status_out;
  if (n > 48) {
    const int np = negf::global_order(n);
    const int grid = negf::sr_global_grid(np);
    if (grid <= 0) return cuda_fail("negf_sgf_sr_f64: occupancy query");
    if (!workspace || workspace_bytes < kCounterBytes + negf::sr_global_ws_bytes(np, grid))
      return fail(NEGF_EINVAL, "negf_sgf_sr_f64: workspace missing or too small (see negf_sgf_workspace_bytes)");
    if (batch == 0) return 0;
    cudaStream_t st = as_stream(stream);
    if (cudaMemsetAsync(workspace, 0, sizeof(unsigned int), st) != cudaSuccess)
      return cuda_fail("negf_sgf_sr_f64: counter reset");
    const int grc = negf::sr_f64_global_launch(a, np, grid,
                                               reinterpret_cast<double2*>(static_cast<char*>(workspace) + kCounterBytes),
                                               reinterpret_cast<unsigned*>(workspace), st);
    if (grc != 0) return cuda_fail("negf_sgf_sr_f64 (global)");
    return 0;
  }
  int rc = negf::sr_f64_launch(a, as_stream(stream));
  if (rc == -2) return fail(NEGF_EUNSUPPORTED, "negf_sgf_sr_f64: block order not built");
  if (rc != 0) return fail(NEGF_ECUDA, negf::last_launch_error());
  return 0;
}

namespace {
int max3(int a, int b, int c) { return a > b ? (a > c ? a : c) : (b > c ? b : c); }
// Persistent grid of the RGF kernel (0 for the 1x1 path, negative on error).
int rgf_grid_for(int np) { return np == 1 ? 0 : negf::rgf_f64_grid(np); }
}  // namespace

size_t negf_rgf_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0) return 0;
  const int nmax = max3(n_dev, n_lead_l, n_lead_r);
  if (nmax > 48) {
    const int gp = negf::global_order(nmax);
    if (gp == 0) return 0;
    const int g = negf::rgf_global_grid(gp);
    if (g <= 0) return 0;
    return kCounterBytes + negf::rgf_global_ws_bytes(gp, n_dev, g);
  }
  const int np = negf::padded_order(nmax);
  if (np == 0) return 0;
  const int grid = rgf_grid_for(np);
  if (grid < 0) return 0;
  return kCounterBytes + (size_t)grid * 2 * n_dev * n_dev * 16;
}

int negf_rgf_transmission_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch, const double* onsite,
                              long long onsite_kstride, long long onsite_lstride, const double* coupling,
                              long long coupling_kstride, long long coupling_lstride, const double* v_left,
                              long long v_left_kstride, const double* v_right, long long v_right_kstride,
                              const double* g_left, long long g_left_pstride, const double* g_right,
                              long long g_right_pstride, const int* k_index, const double* omega,
                              const double* eta_device, const int* lead_status, double* t_out, int* status_out,
                              void* workspace, size_t workspace_bytes, void* stream) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0 || n_layers <= 0 || batch < 0)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_f64: sizes must be positive");
  if (!onsite || !v_left || !v_right || !g_left || !g_right || !omega || !eta_device || !t_out)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_f64: null pointer");
  if (n_layers > 1 && !coupling) return fail(NEGF_EINVAL, "negf_rgf_transmission_f64: null coupling");
  if (onsite_kstride < 0 || onsite_lstride < 0 || coupling_kstride < 0 || coupling_lstride < 0 ||
      v_left_kstride < 0 || v_right_kstride < 0 || g_left_pstride < 0 || g_right_pstride < 0)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_f64: negative stride");
  const int nmax = max3(n_dev, n_lead_l, n_lead_r);
  const bool global = nmax > 48;
  const int np = global ? negf::global_order(nmax) : negf::padded_order(nmax);
  if (np == 0) return fail(NEGF_EUNSUPPORTED, "negf_rgf_transmission_f64: block order above 256");
  const int grid = global ? negf::rgf_global_grid(np) : rgf_grid_for(np);
  if (grid < 0) return cuda_fail("negf_rgf_transmission_f64: occupancy query");
  const size_t need = kCounterBytes + (global ? negf::rgf_global_ws_bytes(np, n_dev, grid)
                                              : (size_t)grid * 2 * n_dev * n_dev * 16);
  if (!workspace || workspace_bytes < need)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_f64: workspace missing or too small");
  if (batch == 0) return 0;
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
  a.counter = reinterpret_cast<unsigned int*>(workspace);
  a.sigma_ws = reinterpret_cast<double2*>(static_cast<char*>(workspace) + kCounterBytes);
  cudaStream_t st = as_stream(stream);
  if (np != 1 && cudaMemsetAsync(workspace, 0, sizeof(unsigned int), st) != cudaSuccess)
    return cuda_fail("negf_rgf_transmission_f64: counter reset");
  int rc = global ? negf::rgf_f64_global_launch(a, np, grid, a.sigma_ws, st) : negf::rgf_f64_launch(a, np, grid, st);
  if (rc == -2) return fail(NEGF_EUNSUPPORTED, "negf_rgf_transmission_f64: block order not built");
  if (rc != 0) return fail(NEGF_ECUDA, negf::last_launch_error());
  return 0;
}

size_t negf_rgf_mixed_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0) return 0;
  const int np = negf::mixed_order(max3(n_dev, n_lead_l, n_lead_r));
  if (np == 0) return 0;
  const int grid = negf::rgf_mixed_grid(np);
  if (grid <= 0) return 0;
  return kCounterBytes + negf::rgf_mixed_ws_bytes(np, n_dev, grid);
}

int negf_rgf_transmission_mixed(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch,
                                const double* onsite, long long onsite_kstride, long long onsite_lstride,
                                const double* coupling, long long coupling_kstride, long long coupling_lstride,
                                const double* v_left, long long v_left_kstride, const double* v_right,
                                long long v_right_kstride, const double* g_left, long long g_left_pstride,
                                const double* g_right, long long g_right_pstride, const int* k_index,
                                const double* omega, const double* eta_device, const int* lead_status,
                                double* t_out, int* status_out, void* workspace, size_t workspace_bytes,
                                void* stream) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0 || n_layers <= 0 || batch < 0)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_mixed: sizes must be positive");
  if (!onsite || !v_left || !v_right || !g_left || !g_right || !omega || !eta_device || !t_out)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_mixed: null pointer");
  if (n_layers > 1 && !coupling) return fail(NEGF_EINVAL, "negf_rgf_transmission_mixed: null coupling");
  if (onsite_kstride < 0 || onsite_lstride < 0 || coupling_kstride < 0 || coupling_lstride < 0 ||
      v_left_kstride < 0 || v_right_kstride < 0 || g_left_pstride < 0 || g_right_pstride < 0)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_mixed: negative stride");
  const int np = negf::mixed_order(max3(n_dev, n_lead_l, n_lead_r));
  if (np == 0) return fail(NEGF_EUNSUPPORTED, "negf_rgf_transmission_mixed: block order above 256");
  const int grid = negf::rgf_mixed_grid(np);
  if (grid <= 0) return cuda_fail("negf_rgf_transmission_mixed: occupancy query");
  if (!workspace || workspace_bytes < kCounterBytes + negf::rgf_mixed_ws_bytes(np, n_dev, grid))
    return fail(NEGF_EINVAL, "negf_rgf_transmission_mixed: workspace missing or too small");
  if (batch == 0) return 0;
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
  a.counter = reinterpret_cast<unsigned int*>(workspace);
  a.sigma_ws = nullptr;
  cudaStream_t st = as_stream(stream);
  if (cudaMemsetAsync(workspace, 0, sizeof(unsigned int), st) != cudaSuccess)
    return cuda_fail("negf_rgf_transmission_mixed: counter reset");
  if (negf::rgf_mixed_launch(a, np, grid, static_cast<char*>(workspace) + kCounterBytes, st) != 0)
    return cuda_fail("negf_rgf_transmission_mixed");
  return 0;
}

size_t negf_rgf_refined_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r, int n_layers) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0 || n_layers <= 0) return 0;
  const int np = negf::mixed_order(max3(n_dev, n_lead_l, n_lead_r));
  if (np == 0) return 0;
  const int grid = negf::rgf_refine_grid(np);
  if (grid <= 0) return 0;
  return kCounterBytes + negf::rgf_refine_ws_bytes(np, n_dev, n_layers, grid);
}

int negf_rgf_transmission_refined(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch,
                                  const double* onsite, long long onsite_kstride, long long onsite_lstride,
                                  const double* coupling, long long coupling_kstride, long long coupling_lstride,
                                  const double* v_left, long long v_left_kstride, const double* v_right,
                                  long long v_right_kstride, const double* g_left, long long g_left_pstride,
                                  const double* g_right, long long g_right_pstride, const int* k_index,
                                  const double* omega, const double* eta_device, const int* lead_status,
                                  double tol, int max_steps, double* t_out, int* status_out, int* steps_out,
                                  void* workspace, size_t workspace_bytes, void* stream) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0 || n_layers <= 0 || batch < 0)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_refined: sizes must be positive");
  if (!onsite || !v_left || !v_right || !g_left || !g_right || !omega || !eta_device || !t_out)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_refined: null pointer");
  if (n_layers > 1 && !coupling) return fail(NEGF_EINVAL, "negf_rgf_transmission_refined: null coupling");
  if (onsite_kstride < 0 || onsite_lstride < 0 || coupling_kstride < 0 || coupling_lstride < 0 ||
      v_left_kstride < 0 || v_right_kstride < 0 || g_left_pstride < 0 || g_right_pstride < 0)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_refined: negative stride");
  if (!(tol > 0.0) || max_steps <= 0)
    return fail(NEGF_EINVAL, "negf_rgf_transmission_refined: tol and max_steps must be positive");
  const int np = negf::mixed_order(max3(n_dev, n_lead_l, n_lead_r));
  if (np == 0) return fail(NEGF_EUNSUPPORTED, "negf_rgf_transmission_refined: block order above 256");
  const int grid = negf::rgf_refine_grid(np);
  if (grid <= 0) return cuda_fail("negf_rgf_transmission_refined: occupancy query");
  if (!workspace || workspace_bytes < kCounterBytes + negf::rgf_refine_ws_bytes(np, n_dev, n_layers, grid))
    return fail(NEGF_EINVAL, "negf_rgf_transmission_refined: workspace missing or too small");
  if (batch == 0) return 0;
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
  a.counter = reinterpret_cast<unsigned int*>(workspace);
  a.sigma_ws = nullptr;
  cudaStream_t st = as_stream(stream);
  if (cudaMemsetAsync(workspace, 0, sizeof(unsigned int), st) != cudaSuccess)
    return cuda_fail("negf_rgf_transmission_refined: counter reset");
  if (negf::rgf_refine_launch(a, np, grid, static_cast<char*>(workspace) + kCounterBytes, tol, max_steps,
                              steps_out, st) != 0)
    return cuda_fail("negf_rgf_transmission_refined");
  return 0;
}

int negf_cgemm_tf32x3(int n, int batch, const float* a, const float* b, float* c, int conj_a, int conj_b,
                      int* status_out, void* stream) {
  if (batch < 0 || n <= 0) return fail(NEGF_EINVAL, "negf_cgemm_tf32x3: sizes must be positive");
  if (n % 16 != 0 || n > 128)
    return fail(NEGF_EUNSUPPORTED, "negf_cgemm_tf32x3: n must be a multiple of 16 up to 128");
  if (!a || !b || !c) return fail(NEGF_EINVAL, "negf_cgemm_tf32x3: null pointer");
  if (batch == 0) return 0;
  if (negf::tc_cgemm_launch(n, batch, reinterpret_cast<const float2*>(a), reinterpret_cast<const float2*>(b),
                            reinterpret_cast<float2*>(c), conj_a, conj_b, status_out, as_stream(stream)) != 0)
    return cuda_fail("negf_cgemm_tf32x3");
  return 0;
}

int negf_set_fp32_product_path(int n, int path) {
  if (n <= 0 || n > 256 || path < -1 || path > 1)
    return fail(NEGF_EINVAL, "negf_set_fp32_product_path: order 1..256 and path -1, 0 or 1");
  const int np = negf::mixed_order(n);
  const int rc = negf::set_fp32_product_path(np, path);
  if (rc == -2) return fail(NEGF_EUNSUPPORTED, "negf_set_fp32_product_path: tcgen05 tiles for orders up to 128 only");
  if (rc < 0) return fail(NEGF_EINVAL, "negf_set_fp32_product_path: bad order");
  return rc;
}

int negf_batch_max_grid(int max_order, int precision, int blocks_per_sm) {
  if (max_order <= 0 || max_order > 256 || (precision != 0 && precision != 1)) return 0;
  if (blocks_per_sm != 1 && blocks_per_sm != 2) return 0;
  const int g = negf::batch_max_grid((max_order + 15) / 16 * 16, precision, blocks_per_sm);
  return g > 0 ? g : 0;
}

size_t negf_batch_system_bytes(void) { return sizeof(NegfBatchSystem); }

size_t negf_batch_workspace_bytes(int max_order, int precision, int blocks_per_sm, int grid) {
  const int gmax = negf_batch_max_grid(max_order, precision, blocks_per_sm);
  if (gmax <= 0) return 0;
  const int g = (grid <= 0 || grid > gmax) ? gmax : grid;
  return kCounterBytes + negf::batch_ws_bytes((max_order + 15) / 16 * 16, g);
}

int negf_batch_transmission(const NegfBatchSystem* systems, int n_systems, int max_order, const int* item_system,
                            const int* item_k, const double* item_omega, int n_items, double tol, int maxiter,
                            int precision, int blocks_per_sm, int grid, double* t_out, int* status_out,
                            int* iters_out, void* workspace, size_t workspace_bytes, void* stream) {
  if (n_systems <= 0 || n_items < 0) return fail(NEGF_EINVAL, "negf_batch_transmission: bad sizes");
  if (!systems || !item_system || !item_k || !item_omega || !t_out)
    return fail(NEGF_EINVAL, "negf_batch_transmission: null pointer");
  if (max_order <= 0 || max_order > 256)
    return fail(NEGF_EUNSUPPORTED, "negf_batch_transmission: max_order must be in 1..256");
  if (precision != 0 && precision != 1) return fail(NEGF_EINVAL, "negf_batch_transmission: precision must be 0 or 1");
  if (maxiter <= 0 || !(tol > 0.0)) return fail(NEGF_EINVAL, "negf_batch_transmission: maxiter and tol must be positive");
  if (blocks_per_sm != 1 && blocks_per_sm != 2)
    return fail(NEGF_EINVAL, "negf_batch_transmission: blocks_per_sm must be 1 or 2");
  const int gmax = negf_batch_max_grid(max_order, precision, blocks_per_sm);
  if (gmax <= 0) return cuda_fail("negf_batch_transmission: occupancy query");
  if (grid > gmax) return fail(NEGF_EINVAL, "negf_batch_transmission: grid above negf_batch_max_grid");
  const int g = grid <= 0 ? gmax : grid;
  const int npmax = (max_order + 15) / 16 * 16;
  if (!workspace || workspace_bytes < kCounterBytes + negf::batch_ws_bytes(npmax, g))
    return fail(NEGF_EINVAL, "negf_batch_transmission: workspace missing or too small");
  if (n_items == 0) return 0;
  cudaStream_t st = as_stream(stream);
  if (cudaMemsetAsync(workspace, 0, sizeof(unsigned int), st) != cudaSuccess)
    return cuda_fail("negf_batch_transmission: counter reset");
  if (negf::batch_launch(systems, n_systems, item_system, item_k, item_omega, n_items, tol, maxiter, t_out,
                         status_out, iters_out, npmax, precision, blocks_per_sm, g, workspace,
                         static_cast<char*>(workspace) + kCounterBytes, st) != 0)
    return cuda_fail("negf_batch_transmission");
  return 0;
}

size_t negf_device_green_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r, int n_layers) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0 || n_layers <= 0) return 0;
  const int nmax = max3(n_dev, n_lead_l, n_lead_r);
  if (nmax > 256) return 0;
  const int np = (nmax + 15) / 16 * 16;
  const int grid = negf::full_grid(np);
  if (grid <= 0) return 0;
  return kCounterBytes + negf::full_ws_bytes(np, n_dev, n_layers, grid);
}

int negf_device_green_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch, const double* onsite,
                          long long onsite_kstride, long long onsite_lstride, const double* coupling,
                          long long coupling_kstride, long long coupling_lstride, const double* v_left,
                          long long v_left_kstride, const double* v_right, long long v_right_kstride,
                          const double* g_left, long long g_left_pstride, const double* g_right,
                          long long g_right_pstride, const int* k_index, const double* omega,
                          const double* eta_device, const int* lead_status, double* g_out, double* sigma_l_out,
                          double* sigma_r_out, int* status_out, void* workspace, size_t workspace_bytes,
                          void* stream) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0 || n_layers <= 0 || batch < 0)
    return fail(NEGF_EINVAL, "negf_device_green_f64: sizes must be positive");
  if (!onsite || !v_left || !v_right || !g_left || !g_right || !omega || !eta_device || !g_out || !sigma_l_out ||
      !sigma_r_out || (n_layers > 1 && !coupling))
    return fail(NEGF_EINVAL, "negf_device_green_f64: null pointer");
  if (onsite_kstride < 0 || onsite_lstride < 0 || coupling_kstride < 0 || coupling_lstride < 0 ||
      v_left_kstride < 0 || v_right_kstride < 0 || g_left_pstride < 0 || g_right_pstride < 0)
    return fail(NEGF_EINVAL, "negf_device_green_f64: negative stride");
  const int nmax = max3(n_dev, n_lead_l, n_lead_r);
  if (nmax > 256) return fail(NEGF_EUNSUPPORTED, "negf_device_green_f64: block order above 256");
  const int np = (nmax + 15) / 16 * 16;
  const int grid = negf::full_grid(np);
  if (grid <= 0) return cuda_fail("negf_device_green_f64: occupancy query");
  if (!workspace || workspace_bytes < kCounterBytes + negf::full_ws_bytes(np, n_dev, n_layers, grid))
    return fail(NEGF_EINVAL, "negf_device_green_f64: workspace missing or too small");
  if (batch == 0) return 0;
  negf::FullArgs fa;
  negf::RgfArgs& a = fa.r;
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
  a.T_out = nullptr;
  a.status_out = status_out;
  a.counter = reinterpret_cast<unsigned int*>(workspace);
  a.sigma_ws = nullptr;
  fa.G = reinterpret_cast<double2*>(g_out);
  fa.sigL_out = reinterpret_cast<double2*>(sigma_l_out);
  fa.sigR_out = reinterpret_cast<double2*>(sigma_r_out);
  cudaStream_t st = as_stream(stream);
  if (cudaMemsetAsync(workspace, 0, sizeof(unsigned int), st) != cudaSuccess)
    return cuda_fail("negf_device_green_f64: counter reset");
  if (negf::full_f64_launch(fa, np, grid, reinterpret_cast<double2*>(static_cast<char*>(workspace) + kCounterBytes),
                            st) != 0)
    return cuda_fail("negf_device_green_f64");
  return 0;
}

size_t negf_adjoint_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r, int n_layers) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0 || n_layers <= 0) return 0;
  const int nmax = max3(n_dev, n_lead_l, n_lead_r);
  if (nmax > 256) return 0;
  const int np = (nmax + 15) / 16 * 16;
  const int grid = negf::grad_grid(np);
  if (grid <= 0) return 0;
  return kCounterBytes + negf::grad_ws_bytes(np, n_dev, n_layers, grid);
}

}  // extern "C"

static int fail2(int code, const char* name, const char* what) {
  char msg[256];
  std::snprintf(msg, sizeof(msg), "%s: %s", name, what);
  return fail(code, msg);
}
static int cuda_fail2(const char* name, const char* what) {
  char msg[256];
  std::snprintf(msg, sizeof(msg), "%s: %s", name, what);
  return cuda_fail(msg);
}

// Shared body of negf_rgf_adjoint_f64 and negf_rgf_adjoint_sigma_f64 (which
// also writes the per-point self-energy adjoints when sig_adj_l/r are set).
static int rgf_adjoint_common(const char* name, int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch,
                              const double* onsite, long long onsite_kstride, long long onsite_lstride,
                              const double* coupling, long long coupling_kstride, long long coupling_lstride,
                              const double* v_left, long long v_left_kstride, const double* v_right,
                              long long v_right_kstride, const double* g_left, long long g_left_pstride,
                              const double* g_right, long long g_right_pstride, const int* k_index,
                              const double* omega, const double* eta_device, const int* lead_status,
                              const double* weight, double* grad_onsite, double* grad_coupling, double* t_out,
                              int* status_out, void* workspace, size_t workspace_bytes, void* stream,
                              double* sig_adj_l, double* sig_adj_r, int per_point) {
  if (n_dev <= 0 || n_lead_l <= 0 || n_lead_r <= 0 || n_layers <= 0 || batch < 0)
    return fail2(NEGF_EINVAL, name, "sizes must be positive");
  if (!onsite || !v_left || !v_right || !g_left || !g_right || !omega || !eta_device || !t_out || !weight ||
      !grad_onsite || (n_layers > 1 && (!coupling || !grad_coupling)))
    return fail2(NEGF_EINVAL, name, "null pointer");
  if (onsite_kstride < 0 || onsite_lstride < 0 || coupling_kstride < 0 || coupling_lstride < 0 ||
      v_left_kstride < 0 || v_right_kstride < 0 || g_left_pstride < 0 || g_right_pstride < 0)
    return fail2(NEGF_EINVAL, name, "negative stride");
  const int nmax = max3(n_dev, n_lead_l, n_lead_r);
  if (nmax > 256) return fail2(NEGF_EUNSUPPORTED, name, "block order above 256");
  const int np = (nmax + 15) / 16 * 16;
  const int grid = negf::grad_grid(np);
  if (grid <= 0) return cuda_fail2(name, "occupancy query");
  if (!workspace || workspace_bytes < kCounterBytes + negf::grad_ws_bytes(np, n_dev, n_layers, grid))
    return fail2(NEGF_EINVAL, name, "workspace missing or too small");
  if (batch == 0) return 0;
  negf::GradArgs ga;
  negf::RgfArgs& a = ga.r;
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
  a.counter = reinterpret_cast<unsigned int*>(workspace);
  a.sigma_ws = nullptr;
  ga.weight = weight;
  ga.grad_d = reinterpret_cast<double2*>(grad_onsite);
  ga.grad_c = reinterpret_cast<double2*>(grad_coupling ? grad_coupling : grad_onsite);
  ga.sig_adj_l = reinterpret_cast<double2*>(sig_adj_l);
  ga.sig_adj_r = reinterpret_cast<double2*>(sig_adj_r);
  ga.per_point = per_point;
  cudaStream_t st = as_stream(stream);
  if (cudaMemsetAsync(workspace, 0, sizeof(unsigned int), st) != cudaSuccess)
    return cuda_fail2(name, "counter reset");
  const int rc = negf::grad_f64_launch(ga, np, grid,
                                       reinterpret_cast<double2*>(static_cast<char*>(workspace) + kCounterBytes), st);
  if (rc != 0) return cuda_fail2(name, "launch");
  return 0;
}

extern "C" {

int negf_rgf_adjoint_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch, const double* onsite,
                         long long onsite_kstride, long long onsite_lstride, const double* coupling,
                         long long coupling_kstride, long long coupling_lstride, const double* v_left,
                         long long v_left_kstride, const double* v_right, long long v_right_kstride,
                         const double* g_left, long long g_left_pstride, const double* g_right,
                         long long g_right_pstride, const int* k_index, const double* omega,
                         const double* eta_device, const int* lead_status, const double* weight, double* grad_onsite,
                         double* grad_coupling, double* t_out, int* status_out, void* workspace,
                         size_t workspace_bytes, void* stream) {
  return rgf_adjoint_common("negf_rgf_adjoint_f64", n_dev, n_lead_l, n_lead_r, n_layers, batch, onsite,
                            onsite_kstride, onsite_lstride, coupling, coupling_kstride, coupling_lstride, v_left,
                            v_left_kstride, v_right, v_right_kstride, g_left, g_left_pstride, g_right,
                            g_right_pstride, k_index, omega, eta_device, lead_status, weight, grad_onsite,
                            grad_coupling, t_out, status_out, workspace, workspace_bytes, stream, nullptr, nullptr, 0);
}

int negf_rgf_adjoint_sigma_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch, const double* onsite,
                               long long onsite_kstride, long long onsite_lstride, const double* coupling,
                               long long coupling_kstride, long long coupling_lstride, const double* v_left,
                               long long v_left_kstride, const double* v_right, long long v_right_kstride,
                               const double* g_left, long long g_left_pstride, const double* g_right,
                               long long g_right_pstride, const int* k_index, const double* omega,
                               const double* eta_device, const int* lead_status, const double* weight,
                               double* grad_onsite, double* grad_coupling, double* sigma_adj_left,
                               double* sigma_adj_right, double* t_out, int* status_out, void* workspace,
                               size_t workspace_bytes, void* stream) {
  if (!sigma_adj_left && !sigma_adj_right)
    return fail(NEGF_EINVAL, "negf_rgf_adjoint_sigma_f64: no self-energy adjoint output");
  return rgf_adjoint_common("negf_rgf_adjoint_sigma_f64", n_dev, n_lead_l, n_lead_r, n_layers, batch, onsite,
                            onsite_kstride, onsite_lstride, coupling, coupling_kstride, coupling_lstride, v_left,
                            v_left_kstride, v_right, v_right_kstride, g_left, g_left_pstride, g_right,
                            g_right_pstride, k_index, omega, eta_device, lead_status, weight, grad_onsite,
                            grad_coupling, t_out, status_out, workspace, workspace_bytes, stream, sigma_adj_left,
                            sigma_adj_right, 0);
}

int negf_rgf_adjoint_points_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch, const double* onsite,
                                long long onsite_kstride, long long onsite_lstride, const double* coupling,
                                long long coupling_kstride, long long coupling_lstride, const double* v_left,
                                long long v_left_kstride, const double* v_right, long long v_right_kstride,
                                const double* g_left, long long g_left_pstride, const double* g_right,
                                long long g_right_pstride, const int* k_index, const double* omega,
                                const double* eta_device, const int* lead_status, const double* weight,
                                double* grad_onsite, double* grad_coupling, double* sigma_adj_left,
                                double* sigma_adj_right, double* t_out, int* status_out, void* workspace,
                                size_t workspace_bytes, void* stream) {
  return rgf_adjoint_common("negf_rgf_adjoint_points_f64", n_dev, n_lead_l, n_lead_r, n_layers, batch, onsite,
                            onsite_kstride, onsite_lstride, coupling, coupling_kstride, coupling_lstride, v_left,
                            v_left_kstride, v_right, v_right_kstride, g_left, g_left_pstride, g_right,
                            g_right_pstride, k_index, omega, eta_device, lead_status, weight, grad_onsite,
                            grad_coupling, t_out, status_out, workspace, workspace_bytes, stream, sigma_adj_left,
                            sigma_adj_right, 1);
}

size_t negf_sgf_adjoint_workspace_bytes(int n_lead, int n_dev) {
  if (n_lead <= 0 || n_dev <= 0 || n_lead > 256 || n_dev > 256) return 0;
  const int np = (max3(n_lead, n_dev, 1) + 15) / 16 * 16;
  const int grid = negf::sgf_adj_grid(np);
  if (grid <= 0) return 0;
  return kCounterBytes + negf::sgf_adj_ws_bytes(np, grid);
}

static int sgf_adjoint_common(const char* name, int per_point, int n_lead, int n_dev, int batch,
                              const double* h01, const double* h10,
                         long long lead_stride, const double* v, long long v_kstride, const double* g,
                         long long g_pstride, const double* sigma_adj, const int* k_index, const int* lead_status,
                         double tol, int maxiter, double* grad_h00, double* grad_h01, double* grad_h10,
                         double* grad_v, int* iters_out, int* status_out, void* workspace, size_t workspace_bytes,
                         void* stream) {
  if (n_lead <= 0 || n_dev <= 0 || batch < 0)
    return fail2(NEGF_EINVAL, name, "sizes must be positive");
  if (!h01 || !v || !g || !sigma_adj || !grad_h00 || !grad_h01 || !grad_v || (h10 && !grad_h10))
    return fail2(NEGF_EINVAL, name, "null pointer");
  if (lead_stride < 0 || v_kstride < 0 || g_pstride < 0)
    return fail2(NEGF_EINVAL, name, "negative stride");
  if (maxiter <= 0 || !(tol > 0.0)) return fail2(NEGF_EINVAL, name, "maxiter and tol must be positive");
  if (n_lead > 256 || n_dev > 256) return fail2(NEGF_EUNSUPPORTED, name, "block order above 256");
  const int np = (max3(n_lead, n_dev, 1) + 15) / 16 * 16;
  const int grid = negf::sgf_adj_grid(np);
  if (grid <= 0) return cuda_fail2(name, "occupancy query");
  if (!workspace || workspace_bytes < kCounterBytes + negf::sgf_adj_ws_bytes(np, grid))
    return fail2(NEGF_EINVAL, name, "workspace missing or too small");
  if (batch == 0) return 0;
  negf::SgfAdjArgs sa;
  sa.nl = n_lead;
  sa.n = n_dev;
  sa.batch = batch;
  sa.h01 = reinterpret_cast<const double2*>(h01);
  sa.h10 = reinterpret_cast<const double2*>(h10);
  sa.lead_stride = lead_stride;
  sa.V = reinterpret_cast<const double2*>(v);
  sa.v_ks = v_kstride;
  sa.g = reinterpret_cast<const double2*>(g);
  sa.g_ps = g_pstride;
  sa.xs = reinterpret_cast<const double2*>(sigma_adj);
  sa.kidx = k_index;
  sa.lead_status = lead_status;
  sa.tol = tol;
  sa.maxiter = maxiter;
  sa.grad_h00 = reinterpret_cast<double2*>(grad_h00);
  sa.grad_h01 = reinterpret_cast<double2*>(grad_h01);
  sa.grad_h10 = h10 ? reinterpret_cast<double2*>(grad_h10) : nullptr;
  sa.grad_v = reinterpret_cast<double2*>(grad_v);
  sa.per_point = per_point;
  sa.iters_out = iters_out;
  sa.status_out = status_out;
  sa.counter = reinterpret_cast<unsigned*>(workspace);
  cudaStream_t st = as_stream(stream);
  if (cudaMemsetAsync(workspace, 0, sizeof(unsigned), st) != cudaSuccess)
    return cuda_fail2(name, "counter reset");
  if (negf::sgf_adj_launch(sa, np, grid, reinterpret_cast<double2*>(static_cast<char*>(workspace) + kCounterBytes),
                           st) != 0)
    return cuda_fail2(name, "launch");
  return 0;
}

int negf_sgf_adjoint_f64(int n_lead, int n_dev, int batch, const double* h01, const double* h10,
                         long long lead_stride, const double* v, long long v_kstride, const double* g,
                         long long g_pstride, const double* sigma_adj, const int* k_index, const int* lead_status,
                         double tol, int maxiter, double* grad_h00, double* grad_h01, double* grad_h10,
                         double* grad_v, int* iters_out, int* status_out, void* workspace, size_t workspace_bytes,
                         void* stream) {
  return sgf_adjoint_common("negf_sgf_adjoint_f64", 0, n_lead, n_dev, batch, h01, h10, lead_stride, v, v_kstride, g,
                            g_pstride, sigma_adj, k_index, lead_status, tol, maxiter, grad_h00, grad_h01, grad_h10,
                            grad_v, iters_out, status_out, workspace, workspace_bytes, stream);
}

int negf_sgf_adjoint_points_f64(int n_lead, int n_dev, int batch, const double* h01, const double* h10,
                                long long lead_stride, const double* v, long long v_kstride, const double* g,
                                long long g_pstride, const double* sigma_adj, const int* k_index,
                                const int* lead_status, double tol, int maxiter, double* grad_h00, double* grad_h01,
                                double* grad_h10, double* grad_v, int* iters_out, int* status_out, void* workspace,
                                size_t workspace_bytes, void* stream) {
  return sgf_adjoint_common("negf_sgf_adjoint_points_f64", 1, n_lead, n_dev, batch, h01, h10, lead_stride, v,
                            v_kstride, g, g_pstride, sigma_adj, k_index, lead_status, tol, maxiter, grad_h00,
                            grad_h01, grad_h10, grad_v, iters_out, status_out, workspace, workspace_bytes, stream);
}

int negf_kmoments_f64(const double* t, int n_omega, int n_k, double* t_mean, double* t2_mean, void* stream) {
  if (n_omega < 0 || n_k <= 0 || !t || !t_mean || !t2_mean) return fail(NEGF_EINVAL, "negf_kmoments_f64: bad argument");
  if (negf::kmoments_launch(t, n_omega, n_k, t_mean, t2_mean, as_stream(stream)) != 0)
    return cuda_fail("negf_kmoments_f64");
  return 0;
}

int negf_fcs_cumulants_f64(const double* omega_rad_s, const double* t_mean, const double* t2_mean, int n_omega,
                           double temp_left, double temp_right, double* c_out, void* stream) {
  if (n_omega < 2 || !omega_rad_s || !t_mean || !t2_mean || !c_out)
    return fail(NEGF_EINVAL, "negf_fcs_cumulants_f64: bad argument");
  if (!(temp_left > 0.0) || !(temp_right > 0.0))
    return fail(NEGF_EINVAL, "negf_fcs_cumulants_f64: temperature must be positive in Kelvin");
  if (negf::fcs_launch(omega_rad_s, t_mean, t2_mean, n_omega, temp_left, temp_right, c_out, as_stream(stream)) != 0)
    return cuda_fail("negf_fcs_cumulants_f64");
  return 0;
}

int negf_heat_current_f64(const double* omega_rad_s, const double* t, int n_omega, int n_spectra, double temp_left,
                          double temp_right, double* j_out, void* stream) {
  if (n_omega < 2 || n_spectra < 0 || !omega_rad_s || !t || !j_out)
    return fail(NEGF_EINVAL, "negf_heat_current_f64: bad argument");
  if (!(temp_left > 0.0) || !(temp_right > 0.0))
    return fail(NEGF_EINVAL, "negf_heat_current_f64: temperatures must be positive in Kelvin");
  if (negf::heat_current_launch(omega_rad_s, t, n_omega, n_spectra, temp_left, temp_right, j_out, as_stream(stream)) != 0)
    return cuda_fail("negf_heat_current_f64");
  return 0;
}

int negf_kavg_f64(const double* t, int n_omega, int n_k, double* t_mean, void* stream) {
  if (n_omega < 0 || n_k <= 0 || !t || !t_mean) return fail(NEGF_EINVAL, "negf_kavg_f64: bad argument");
  if (negf::kavg_launch(t, n_omega, n_k, t_mean, as_stream(stream)) != 0) return cuda_fail("negf_kavg_f64");
  return 0;
}

int negf_kappa_f64(const double* omega, const double* t_mean, int n_omega, const double* temperatures, int n_temps,
                   double omega_unit_rad_s, double* kappa_out, void* stream) {
  if (n_omega < 2 || n_temps < 0 || !omega || !t_mean || !temperatures || !kappa_out)
    return fail(NEGF_EINVAL, "negf_kappa_f64: bad argument");
  if (negf::kappa_launch(omega, t_mean, n_omega, temperatures, n_temps, omega_unit_rad_s, kappa_out,
                         as_stream(stream)) != 0)
    return cuda_fail("negf_kappa_f64");
  return 0;
}

}  // extern "C"
