// Internal launch interface of the FP64 kernels (not part of the C-ABI).
#pragma once
#include <cuda_runtime.h>

struct NegfBatchSystem;  // include/negf_b200.h

namespace negf {

// Sancho-Rubio over a batch of points; complex matrices are interleaved
// (re, im) double pairs, row-major, order n.
struct SrArgs {
  int n, batch;
  const double2* h00;
  const double2* h01;
  const double2* h10;      // nullptr: d10 = d01^H
  long long lead_stride;   // complex elements between consecutive lead sets
  const int* kidx;         // [batch] lead-set index per point (nullptr: set 0)
  const double* omega;     // [batch]
  const double* eta;       // [batch]
  double tol;
  int maxiter;
  double2* g_out;          // [batch][n][n] or nullptr
  double* dos_out;         // [batch] or nullptr
  int* iters_out;          // [batch] or nullptr
  int* status_out;         // [batch] or nullptr
};

// Device solve + transmission over a batch of points.
struct RgfArgs {
  int n, nl, nr, L, batch;
  const double2* D;  long long d_ks, d_ls;    // onsite block (k, l) at D + k*d_ks + l*d_ls
  const double2* C;  long long c_ks, c_ls;    // coupling block (k, l) between layers l and l+1
  const double2* VL; long long vl_ks;         // [.][n][nl] device-to-left-lead coupling
  const double2* VR; long long vr_ks;         // [.][n][nr]
  const double2* gL; long long gl_ps;         // per-point left surface GF, stride per point
  const double2* gR; long long gr_ps;
  const int* kidx;
  const double* omega;
  const double* eta_dev;
  const int* lead_status;   // [batch] or nullptr; nonzero skips the point
  double* T_out;            // [batch]
  int* status_out;          // [batch] or nullptr
  double2* sigma_ws;        // [grid][2][n][n] scratch
  unsigned int* counter;    // zeroed work counter
};

// Adjoint of the device solve: RgfArgs plus per-point weights and the
// per-k accumulators of the adjoint blocks.
struct GradArgs {
  RgfArgs r;
  const double* weight;  // [batch] dKappa/dT of each point
  double2* grad_d;       // [K][L][n][n]    += weight X_ii
  double2* grad_c;       // [K][L-1][n][n]  += weight (X_{i+1,i} + X_{i,i+1}^H)
  double2* sig_adj_l;    // [batch][n][n] or nullptr: weight dT/dSigma_L (X_00 + i G Gamma_R G^H)
  double2* sig_adj_r;    // [batch][n][n] or nullptr: weight dT/dSigma_R (X_{L-1,L-1} + i G^H Gamma_L G)
  int per_point;         // 1: grad_d / grad_c are [batch][..] and each point stores its own blocks
};

// Adjoint of the surface GF fixed point g = (z - H00 - H01 g H10)^-1 and of
// Sigma = V g V^H, per point, accumulated per lead set k.
struct SgfAdjArgs {
  int nl, n, batch;        // lead order, device order
  const double2* h01;
  const double2* h10;      // nullptr: H10 = H01^H (its gradient is folded into grad_h01)
  long long lead_stride;   // complex elements between lead sets
  const double2* V;        // [.][n][nl] device-to-lead coupling of this lead
  long long v_ks;
  const double2* g;        // [batch][nl][nl] surface GFs
  long long g_ps;
  const double2* xs;       // [batch][n][n] weighted dT/dSigma (convention dT = 2 Re Tr[dSigma X])
  const int* kidx;
  const int* lead_status;  // nonzero: skip the point
  double tol;
  int maxiter;
  double2* grad_h00;       // [K][nl][nl] += X-convention adjoints
  double2* grad_h01;
  double2* grad_h10;       // nullptr when h10 is nullptr
  double2* grad_v;         // [K|1][nl][n]
  int per_point;           // 1: the four gradients are [batch][..] and each point stores its own
  int* iters_out;
  int* status_out;
  unsigned* counter;
};

// Full device Green's function: RgfArgs plus the outputs.
struct FullArgs {
  RgfArgs r;
  double2* G;         // [batch][L n][L n]
  double2* sigL_out;  // [batch][n][n]
  double2* sigR_out;  // [batch][n][n]
};

int padded_order(int n);
const char* last_launch_error();  // message of the last failed launch on this thread
// Records `msg` as the text negf_last_error() returns on this host thread and
// returns `code`; for entry points defined outside negf_capi.cu.
int record_error(int code, const char* msg);
int sr_f64_launch(const SrArgs& a, cudaStream_t st);
// Padded order np = padded_order(max(n, nl, nr)) selects the kernel variant.
int rgf_f64_grid(int np);  // persistent grid size (blocks), 0 for the 1x1 path
int rgf_f64_launch(const RgfArgs& a, int np, int grid, cudaStream_t st);
// Block orders 49..256 (padded to a multiple of 16): global-memory workspace kernels.
int global_order(int n);  // padded order for n > 48, 0 if unsupported
int sr_global_grid(int np);
int rgf_global_grid(int np);
size_t sr_global_ws_bytes(int np, int grid);
size_t rgf_global_ws_bytes(int np, int n, int grid);
int sr_f64_global_launch(const SrArgs& a, int np, int grid, double2* ws, unsigned* counter, cudaStream_t st);
int rgf_f64_global_launch(const RgfArgs& a, int np, int grid, double2* ws, cudaStream_t st);

// Mixed precision device solve (FP32 sweep, FP64 self-energies and trace), orders 1..256.
int mixed_order(int n);  // padded order (multiple of 16), 0 if unsupported
int rgf_mixed_grid(int np);
size_t rgf_mixed_ws_bytes(int np, int n, int grid);
int rgf_mixed_launch(const RgfArgs& a, int np, int grid, void* ws, cudaStream_t st);

namespace mixed {
bool use_tc(int np);  // tcgen05 products at this padded order (see set_fp32_product_path)
}
// Product tiling of the FP32 sweeps at padded order np: -1 default, 0 mma.sync,
// 1 tcgen05 (np <= 128).  Returns the effective path, -1 bad order, -2 unsupported.
int set_fp32_product_path(int np, int path);
// Refined device solve (FP32 factors, FP64 iterative refinement), orders 1..256.
int rgf_refine_grid(int np);
size_t rgf_refine_ws_bytes(int np, int n, int L, int grid);
int rgf_refine_launch(const RgfArgs& a, int np, int grid, void* ws, double tol, int maxit, int* steps_out,
                      cudaStream_t st);

// Batched complex FP32 products on tcgen05 (negf_tc.cu), n a multiple of 16 up to 128.
int tc_cgemm_launch(int np, int batch, const float2* a, const float2* b, float2* c, int conj_a, int conj_b,
                    int* status, cudaStream_t st);

// Uneven batch (negf_batch.cu).
int batch_max_grid(int npmax, int mixed, int minb);
size_t batch_ws_bytes(int npmax, int grid);
int batch_launch(const ::NegfBatchSystem* sys, int n_systems, const int* item_system, const int* item_k,
                 const double* item_omega, int n_items, double tol, int maxiter, double* t_out, int* status_out,
                 int* iters_out, int npmax, int mixed, int minb, int grid, void* counter, void* ws, cudaStream_t st);

size_t full_ws_bytes(int np, int n, int L, int grid);
int full_grid(int np);
int full_f64_launch(const FullArgs& fa, int np, int grid, double2* ws, cudaStream_t st);

size_t grad_ws_bytes(int np, int n, int L, int grid);
int grad_grid(int np);
int grad_f64_launch(const GradArgs& ga, int np, int grid, double2* ws, cudaStream_t st);

size_t sgf_adj_ws_bytes(int np, int grid);
int sgf_adj_grid(int np);
int sgf_adj_launch(const SgfAdjArgs& sa, int np, int grid, double2* ws, cudaStream_t st);

int heat_current_launch(const double* om, const double* t, int W, int n_spectra, double temp_l, double temp_r,
                        double* out, cudaStream_t st);
int kmoments_launch(const double* T, int W, int K, double* t1, double* t2, cudaStream_t st);
int fcs_launch(const double* om, const double* t1, const double* t2, int W, double temp_l, double temp_r, double* out,
               cudaStream_t st);
int kavg_launch(const double* T, int W, int K, double* tbar, cudaStream_t st);
int kappa_launch(const double* om, const double* tbar, int W, const double* temps, int nT, double unit, double* out,
                 cudaStream_t st);

}  // namespace negf
