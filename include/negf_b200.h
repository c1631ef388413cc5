/*
 * negf_b200.h -- C ABI of libnegfb200.so, the B200 kernels of the
 * per-(omega, k) phonon NEGF path.
 *
 * Conventions
 *  - All array pointers are DEVICE pointers owned by the caller.
 *  - Complex matrices are interleaved (re, im) float64 pairs, row-major.
 *    Strides are counted in complex elements.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are
 *    asynchronous on that stream; nothing is allocated by the library
 *    (the caller provides every workspace) and nothing is synchronised.
 *  - Return value: 0 on success, negative on a launch-level problem
 *    (NEGF_EINVAL bad argument, NEGF_EUNSUPPORTED size not built,
 *    NEGF_ECUDA CUDA error); negf_last_error() describes it.  Numerical
 *    outcomes are per point in `status_out`: NEGF_OK, NEGF_MAXITER,
 *    NEGF_NONFINITE, NEGF_SINGULAR, NEGF_REFINE_FAIL, NEGF_UNSTABLE.
 *
 * Each entry point names the negfpy routine it replaces (paths relative to
 * the negfpy project root).
 */
#ifndef NEGF_B200_H
#define NEGF_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NEGF_B200_ABI_VERSION 1

#define NEGF_OK 0
#define NEGF_MAXITER 1
#define NEGF_NONFINITE 2
#define NEGF_SINGULAR 3
#define NEGF_REFINE_FAIL 4
#define NEGF_BAD_ITEM 5 /* batch item: system, k index or block order out of range */
#define NEGF_UNSTABLE 6 /* decimation: inf/nan arose inside an iteration from finite blocks */

#define NEGF_EINVAL (-1)
#define NEGF_EUNSUPPORTED (-2)
#define NEGF_ECUDA (-3)

/* ABI version (NEGF_B200_ABI_VERSION). */
int negf_get_version(void);

/* Description of the last failing call on this host thread. */
const char* negf_last_error(void);

/* Largest block order the FP64 kernels accept (orders up to 48 run from
 * shared memory, 49..256 from a global-memory workspace). */
int negf_max_order_f64(void);

/* Workspace bytes negf_sgf_sr_f64 needs for block order n (0 on a bad size). */
size_t negf_sgf_workspace_bytes(int n);

/*
 * Batched Sancho-Rubio surface Green's function, FP64.
 * Replaces negfpy core/surface_gf.py:18-81 (surface_gf_sancho_rubio, reached
 * through the dispatcher core/surface_gf.py:254-311 with method
 * "sancho_rubio") and, through dos_out, the trace of core/dos.py:31-61.
 *
 * Point p uses lead set k = k_index[p] (k_index NULL: k = 0), whose blocks
 * are h00/h01/h10 + k*lead_stride (n x n each; h10 NULL means h01^H), and
 * z = (omega[p] + i eta[p])^2.  Outputs (each may be NULL):
 *   g_out[p]      n x n surface Green's function
 *   dos_out[p]    (omega/pi) Re Tr[i (g - g^H)]
 *   iters_out[p]  decimation sweeps taken
 *   status_out[p] NEGF_OK / NEGF_MAXITER / NEGF_NONFINITE / NEGF_SINGULAR
 * workspace: negf_sgf_workspace_bytes(n) bytes (a work counter, and the
 * per-block matrices for n > 48); block orders 1..256.
 */
int negf_sgf_sr_f64(int n, int batch, const double* h00, const double* h01, const double* h10,
                    long long lead_stride, const int* k_index, const double* omega, const double* eta,
                    double tol, int maxiter, double* g_out, double* dos_out, int* iters_out, int* status_out,
                    void* workspace, size_t workspace_bytes, void* stream);

/* Workspace bytes negf_rgf_transmission_f64 needs (0 on a bad size). */
size_t negf_rgf_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r);

/*
 * Batched device solve and transmission, FP64.
 * Replaces negfpy core/negf.py:306-357 (transmission) including
 * core/negf.py:141-250 (system assembly, Sigma = V g V^H at :72-97) and the
 * SuperLU solve at :353, by a recursive Green's function sweep.
 *
 * Point p uses k = k_index[p]; onsite block l is onsite + k*onsite_kstride +
 * l*onsite_lstride, coupling block l (between layers l, l+1; its conjugate
 * transpose sits below the diagonal) is coupling + k*coupling_kstride +
 * l*coupling_lstride.  v_left (n_dev x n_lead_l) and v_right
 * (n_dev x n_lead_r) are the device-to-lead couplings with the contact DOFs
 * of the first / last layer as rows (zero rows elsewhere); their k stride
 * may be 0.  g_left/g_right are per-point surface Green's functions (point
 * stride g_*_pstride; g_right may equal g_left).  lead_status (may be NULL)
 * skips points whose surface GF failed, copying the status.
 * Output: t_out[p] = Re Tr[Gamma_L G_LR Gamma_R G_LR^H] (NaN on failure).
 */
int negf_rgf_transmission_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch,
                              const double* onsite, long long onsite_kstride, long long onsite_lstride,
                              const double* coupling, long long coupling_kstride, long long coupling_lstride,
                              const double* v_left, long long v_left_kstride, const double* v_right,
                              long long v_right_kstride, const double* g_left, long long g_left_pstride,
                              const double* g_right, long long g_right_pstride, const int* k_index,
                              const double* omega, const double* eta_device, const int* lead_status,
                              double* t_out, int* status_out, void* workspace, size_t workspace_bytes,
                              void* stream);

/*
 * Allocation-free form of negf_rgf_transmission_f64, for callers that cannot
 * allocate device memory when they call (a host program that fixed its GPU
 * memory budget and pools at start-up, or a binding from a language without
 * a CUDA allocator).  It has no counterpart in negfpy.  Same arguments and
 * outputs as negf_rgf_transmission_f64 without the workspace: the scratch
 * lives in one static 16 MiB device array per GPU, held until the process
 * exits.  The first call on a device looks up that array's device address
 * (make it before any stream capture).  Calls share the array: calls whose
 * GPU work overlaps race and must not be issued concurrently.  Returns
 * NEGF_EUNSUPPORTED for block orders above 48, which run only from shared
 * memory here (the allocating form runs orders 49..256 on its global-
 * workspace kernels); the persistent grid is capped to what fits the array.
 * NEGF_EINVAL / NEGF_ECUDA as the other entry points, with the message in
 * negf_last_error().  Calls no allocator.
 */
int negf_rgf_transmission_f64_noalloc(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch,
                                      const double* onsite, long long onsite_kstride, long long onsite_lstride,
                                      const double* coupling, long long coupling_kstride,
                                      long long coupling_lstride, const double* v_left, long long v_left_kstride,
                                      const double* v_right, long long v_right_kstride, const double* g_left,
                                      long long g_left_pstride, const double* g_right, long long g_right_pstride,
                                      const int* k_index, const double* omega, const double* eta_device,
                                      const int* lead_status, double* t_out, int* status_out, void* stream);

/* Workspace bytes negf_device_green_f64 needs (0 on a bad size). */
size_t negf_device_green_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r, int n_layers);

/*
 * Full device Green's function, FP64.  Replaces negfpy core/negf.py:253-303
 * (device_green_function, there a dense SuperLU solve against the identity).
 * Same inputs as negf_rgf_transmission_f64 with layer-resolved or shared
 * blocks; per point p it writes
 *   g_out[p]        G = A^-1, (n_layers n_dev)^2, row-major, every block,
 *   sigma_l_out[p]  Sigma_L = V_L g_L V_L^H (n_dev x n_dev, first layer),
 *   sigma_r_out[p]  Sigma_R (n_dev x n_dev, last layer),
 *   status_out[p]   NEGF_* code (g_out is not written for failed points).
 * One left sweep; the diagonal blocks by G_ii = g_i + g_i C_i G_{i+1,i+1}
 * C_i^H g_i and the off-diagonal ones by G_ij = g_i C_i G_{i+1,j},
 * G_ji = G_{j,i+1} C_i^H g_i (i < j).
 */
int negf_device_green_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch, const double* onsite,
                          long long onsite_kstride, long long onsite_lstride, const double* coupling,
                          long long coupling_kstride, long long coupling_lstride, const double* v_left,
                          long long v_left_kstride, const double* v_right, long long v_right_kstride,
                          const double* g_left, long long g_left_pstride, const double* g_right,
                          long long g_right_pstride, const int* k_index, const double* omega,
                          const double* eta_device, const int* lead_status, double* g_out, double* sigma_l_out,
                          double* sigma_r_out, int* status_out, void* workspace, size_t workspace_bytes,
                          void* stream);

/* Workspace bytes negf_rgf_transmission_mixed needs (0 on a bad size). */
size_t negf_rgf_mixed_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r);

/*
 * Batched device solve and transmission in mixed precision: the same
 * arguments, outputs and status codes as negf_rgf_transmission_f64 (the
 * negfpy routines it replaces are those of core/negf.py:72-357).  The contact
 * self-energies, the broadenings and the trace are FP64; the recursive sweep
 * through the layers runs in FP32 (3 x TF32 tensor-core products, FP32
 * Gauss-Jordan).  A point whose FP32 sweep meets a singular or non-finite
 * pivot reports NEGF_SINGULAR / NEGF_NONFINITE so that the caller can
 * re-solve it with negf_rgf_transmission_f64.  Block orders 1..256.
 */
int negf_rgf_transmission_mixed(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch,
                                const double* onsite, long long onsite_kstride, long long onsite_lstride,
                                const double* coupling, long long coupling_kstride, long long coupling_lstride,
                                const double* v_left, long long v_left_kstride, const double* v_right,
                                long long v_right_kstride, const double* g_left, long long g_left_pstride,
                                const double* g_right, long long g_right_pstride, const int* k_index,
                                const double* omega, const double* eta_device, const int* lead_status,
                                double* t_out, int* status_out, void* workspace, size_t workspace_bytes,
                                void* stream);

/* Workspace bytes negf_rgf_transmission_refined needs (0 on a bad size). */
size_t negf_rgf_refined_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r, int n_layers);

/*
 * Batched device solve and transmission with FP64 accuracy from FP32
 * factors: the arguments, outputs and status codes of
 * negf_rgf_transmission_f64 (replacing negfpy core/negf.py:72-357, whose
 * SuperLU solve of A X = E_R, core/negf.py:346-353, this refines), plus
 * tol, max_steps and steps_out.  The block LU factors of A come from an FP32
 * sweep (3 x TF32 tensor-core products, FP32 Gauss-Jordan); the right-contact
 * block column X is then refined: R = E_R - A X in FP64, A d = R solved with
 * the FP32 factors, X += d.  With nu_k = max|d| / max|X| over all blocks
 * after step k, it stops at the first k >= 2 with nu_k^2 / nu_{k-1} <= tol
 * (the next correction predicted from the measured contraction), or when
 * nu_k <= tol.  A point whose correction fails to halve from one step to the
 * next, or that does not converge within max_steps, reports
 * NEGF_REFINE_FAIL; a singular or non-finite FP32 pivot NEGF_SINGULAR /
 * NEGF_NONFINITE.  The caller re-solves those points with
 * negf_rgf_transmission_f64.  Self-energies, broadenings and the trace are
 * FP64.  steps_out[p] (may be NULL): refinement steps taken.  Block orders
 * 1..256.
 */
int negf_rgf_transmission_refined(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch,
                                  const double* onsite, long long onsite_kstride, long long onsite_lstride,
                                  const double* coupling, long long coupling_kstride, long long coupling_lstride,
                                  const double* v_left, long long v_left_kstride, const double* v_right,
                                  long long v_right_kstride, const double* g_left, long long g_left_pstride,
                                  const double* g_right, long long g_right_pstride, const int* k_index,
                                  const double* omega, const double* eta_device, const int* lead_status,
                                  double tol, int max_steps, double* t_out, int* status_out, int* steps_out,
                                  void* workspace, size_t workspace_bytes, void* stream);

/*
 * Batched complex FP32 products on the fifth-generation tensor cores:
 * c[p] = op(a[p]) op(b[p]) for batch independent n x n matrices (complex64,
 * interleaved re, im, row-major, consecutive), op the conjugate transpose
 * when conj_a / conj_b is nonzero.  Each real product is split 3 x TF32
 * (tcgen05.mma kind::tf32, accumulators in Tensor Memory).  No counterpart
 * in negfpy: the building block of the FP32 device sweeps, exposed so that
 * it can be checked on its own.  n a multiple of 16 up to 128 (else
 * NEGF_EUNSUPPORTED).  status_out[p] (may be NULL): NEGF_OK, or
 * NEGF_NONFINITE if the product's completion wait ran out.
 */
int negf_cgemm_tf32x3(int n, int batch, const float* a, const float* b, float* c, int conj_a, int conj_b,
                      int* status_out, void* stream);

/*
 * Product tiling of the FP32 device sweeps (negf_rgf_transmission_mixed,
 * negf_rgf_transmission_refined) for block order n (padded to 16): path 0
 * mma.sync 16 x 16 warp tiles, 1 tcgen05 128 x n tiles (n <= 128, else
 * NEGF_EUNSUPPORTED), -1 back to the default (mma.sync unless NEGF_TC=1 in
 * the environment).  Process-wide; returns the path now in effect (0 or 1).
 * Set it before querying the workspace of the call it is meant for.  No
 * counterpart in negfpy: the autotuner's switch (negfpy_b200.autotune).
 */
int negf_set_fp32_product_path(int n, int path);

/* Workspace bytes negf_rgf_adjoint_f64 needs (0 on a bad size). */
size_t negf_adjoint_workspace_bytes(int n_dev, int n_lead_l, int n_lead_r, int n_layers);

/*
 * Adjoint of the device solve, FP64 (no counterpart in negfpy, which has no
 * derivatives; it differentiates core/negf.py:306-357 with respect to the
 * device blocks).  Same inputs as negf_rgf_transmission_f64 plus weight[p]
 * (e.g. dkappa/dT of the point).  With G = A^-1, Y = Gamma_R G_{0,L-1}^H
 * Gamma_L and X_ji = G_{j,L-1} Y G_{0,i}, it ADDS, for the point's k:
 *   grad_onsite[k][i]   += weight[p] X_ii                  ([K][L][n][n])
 *   grad_coupling[k][i] += weight[p] (X_{i+1,i} + X_{i,i+1}^H)   ([K][L-1][n][n])
 * so that dT = 2 Re sum_i Tr[dD_i X_ii] + 2 Re sum_i Tr[dC_i (...)].  The
 * caller zeroes the accumulators.  T and status as negf_rgf_transmission_f64;
 * nothing is kept between calls (the forward sweeps are recomputed).
 * Block orders 1..256.
 */
int negf_rgf_adjoint_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch, const double* onsite,
                         long long onsite_kstride, long long onsite_lstride, const double* coupling,
                         long long coupling_kstride, long long coupling_lstride, const double* v_left,
                         long long v_left_kstride, const double* v_right, long long v_right_kstride,
                         const double* g_left, long long g_left_pstride, const double* g_right,
                         long long g_right_pstride, const int* k_index, const double* omega,
                         const double* eta_device, const int* lead_status, const double* weight, double* grad_onsite,
                         double* grad_coupling, double* t_out, int* status_out, void* workspace,
                         size_t workspace_bytes, void* stream);

/*
 * negf_rgf_adjoint_f64 that also writes, per point, the weighted adjoint of
 * each contact self-energy (no counterpart in negfpy; it differentiates
 * core/negf.py:72-116, 306-357 with respect to Sigma_L and Sigma_R):
 *   sigma_adj_left[p]  = weight[p] (X_00 + i G Gamma_R G^H)              ([batch][n][n])
 *   sigma_adj_right[p] = weight[p] (X_{L-1,L-1} + i G^H Gamma_L G)
 * with G = G_{0,L-1}, so that dT = 2 Re Tr[dSigma_L sigma_adj_left] + ...
 * (Sigma enters both A and Gamma).  Either output may be NULL, not both.
 * Points that fail are not written (the caller zeroes the outputs).
 * Workspace as negf_rgf_adjoint_f64 (negf_adjoint_workspace_bytes).
 */
int negf_rgf_adjoint_sigma_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch, const double* onsite,
                               long long onsite_kstride, long long onsite_lstride, const double* coupling,
                               long long coupling_kstride, long long coupling_lstride, const double* v_left,
                               long long v_left_kstride, const double* v_right, long long v_right_kstride,
                               const double* g_left, long long g_left_pstride, const double* g_right,
                               long long g_right_pstride, const int* k_index, const double* omega,
                               const double* eta_device, const int* lead_status, const double* weight,
                               double* grad_onsite, double* grad_coupling, double* sigma_adj_left,
                               double* sigma_adj_right, double* t_out, int* status_out, void* workspace,
                               size_t workspace_bytes, void* stream);

/*
 * negf_rgf_adjoint_sigma_f64 with per-point gradient blocks: grad_onsite is
 * [batch][n_layers][n][n] and grad_coupling [batch][n_layers-1][n][n], and
 * point p STORES weight[p] X_ii and weight[p] (X_{i+1,i} + X_{i,i+1}^H) in
 * its own blocks instead of adding them into shared per-k blocks.  Summing
 * the points' blocks per k in a fixed order then gives a gradient that is
 * the same bit for bit from run to run (the FP64 atomic additions of
 * negf_rgf_adjoint_f64 follow the GPU's scheduling).  Points that fail or
 * are skipped are not written (the caller zeroes the outputs).  Both
 * self-energy outputs may be NULL.  Same workspace as negf_rgf_adjoint_f64.
 */
int negf_rgf_adjoint_points_f64(int n_dev, int n_lead_l, int n_lead_r, int n_layers, int batch, const double* onsite,
                                long long onsite_kstride, long long onsite_lstride, const double* coupling,
                                long long coupling_kstride, long long coupling_lstride, const double* v_left,
                                long long v_left_kstride, const double* v_right, long long v_right_kstride,
                                const double* g_left, long long g_left_pstride, const double* g_right,
                                long long g_right_pstride, const int* k_index, const double* omega,
                                const double* eta_device, const int* lead_status, const double* weight,
                                double* grad_onsite, double* grad_coupling, double* sigma_adj_left,
                                double* sigma_adj_right, double* t_out, int* status_out, void* workspace,
                                size_t workspace_bytes, void* stream);

/* Workspace bytes negf_sgf_adjoint_f64 needs (0 on a bad size). */
size_t negf_sgf_adjoint_workspace_bytes(int n_lead, int n_dev);

/*
 * Adjoint of the surface Green's function and of Sigma = V g V^H, FP64 (no
 * counterpart in negfpy; it differentiates the fixed point that
 * core/surface_gf.py:18-81 decimates to, g = (z - H00 - H01 g H10)^-1, and
 * core/negf.py:72-97, Sigma = V g V^H, implicitly: nothing is differentiated
 * through the decimation sweeps).  Per point p with lead set k = k_index[p]:
 * g[p] (n_lead x n_lead, from negf_sgf_sr_f64), the coupling V at
 * v + k*v_kstride (n_dev x n_lead) and sigma_adj[p] (n_dev x n_dev, from
 * negf_rgf_adjoint_sigma_f64).  It solves Lam - Q Lam P = V^H X V with
 * P = g H01, Q = H10 g by doubling (until max(|Q^(2^j)|, |P^(2^j)|) < tol,
 * at most maxiter doublings; iters_out) and ADDS, in the convention
 * dT = 2 Re Tr[dH X]:
 *   grad_h00[k] += g Lam g,  grad_h01[k] += g H10 g Lam g,
 *   grad_h10[k] += g Lam g H01 g      (h10 NULL: H10 = H01^H, and this
 *                                      term's ^H is added to grad_h01),
 *   grad_v[k]   += g V^H X + g^H V^H X^H     ([K or 1][n_lead][n_dev]).
 * The caller zeroes the accumulators.  Status per point: NEGF_MAXITER,
 * NEGF_NONFINITE; points with nonzero lead_status are skipped.  Orders
 * 1..256.
 */
int negf_sgf_adjoint_f64(int n_lead, int n_dev, int batch, const double* h01, const double* h10,
                         long long lead_stride, const double* v, long long v_kstride, const double* g,
                         long long g_pstride, const double* sigma_adj, const int* k_index, const int* lead_status,
                         double tol, int maxiter, double* grad_h00, double* grad_h01, double* grad_h10,
                         double* grad_v, int* iters_out, int* status_out, void* workspace, size_t workspace_bytes,
                         void* stream);

/*
 * negf_sgf_adjoint_f64 with per-point gradients: grad_h00, grad_h01,
 * grad_h10 are [batch][n_lead][n_lead] and grad_v [batch][n_lead][n_dev],
 * and point p STORES its terms in its own slot (summed per k by the caller
 * in a fixed order for a run-to-run reproducible gradient).  Skipped or
 * failed points are not written (the caller zeroes the outputs).  Same
 * workspace as negf_sgf_adjoint_f64.
 */
int negf_sgf_adjoint_points_f64(int n_lead, int n_dev, int batch, const double* h01, const double* h10,
                                long long lead_stride, const double* v, long long v_kstride, const double* g,
                                long long g_pstride, const double* sigma_adj, const int* k_index,
                                const int* lead_status, double tol, int maxiter, double* grad_h00, double* grad_h01,
                                double* grad_h10, double* grad_v, int* iters_out, int* status_out, void* workspace,
                                size_t workspace_bytes, void* stream);

/*
 * One lead/device/lead system of an uneven batch (negf_batch_transmission).
 * Pointers are device pointers to complex128 (interleaved re, im) blocks with
 * the layouts of negf_sgf_sr_f64 and negf_rgf_transmission_f64: lead set k at
 * lead_*_h00/h01/h10 + k*lead_*_kstride (h10 NULL: h01^H), onsite block (k, l)
 * at onsite + k*onsite_kstride + l*onsite_lstride, and so on.  same_leads
 * nonzero: the right lead is the left one (one decimation per item; then
 * n_lead_r must equal n_lead_l).  n_k: number of k sets; items with k outside
 * [0, n_k) report NEGF_BAD_ITEM.
 */
typedef struct NegfBatchSystem {
  int n_dev, n_lead_l, n_lead_r, n_layers, n_k, same_leads;
  const double* onsite;
  long long onsite_kstride, onsite_lstride;
  const double* coupling;
  long long coupling_kstride, coupling_lstride;
  const double* v_left;
  long long v_left_kstride;
  const double* v_right;
  long long v_right_kstride;
  const double* lead_l_h00;
  const double* lead_l_h01;
  const double* lead_l_h10;
  long long lead_l_kstride;
  const double* lead_r_h00;
  const double* lead_r_h01;
  const double* lead_r_h10;
  long long lead_r_kstride;
  double eta, eta_device;
} NegfBatchSystem;

/* Largest persistent grid (blocks) of the batch kernel for systems of block
 * order up to max_order; precision 0 = FP64 device solve, 1 = mixed;
 * blocks_per_sm 1 or 2 selects the kernel variant whose registers are capped
 * for that many resident blocks (0 on a bad argument). */
int negf_batch_max_grid(int max_order, int precision, int blocks_per_sm);

/* Workspace bytes of negf_batch_transmission (grid <= 0: the largest grid). */
size_t negf_batch_workspace_bytes(int max_order, int precision, int blocks_per_sm, int grid);

/* sizeof(NegfBatchSystem), for bindings that lay the table out themselves. */
size_t negf_batch_system_bytes(void);

/*
 * Uneven batch in one persistent launch: item i is system item_system[i] of
 * the device-memory table `systems` at its k set item_k[i] and frequency
 * item_omega[i].  Per item: the lead decimation(s) of negf_sgf_sr_f64 and the
 * device solve of negf_rgf_transmission_f64 (precision 0) or of
 * negf_rgf_transmission_mixed (precision 1), i.e. negfpy core/negf.py:306-357
 * per (system, omega, k).  Items run in the given order, one block each, taken
 * from a work counter: order them by decreasing cost for a short tail.
 * Outputs per item: t_out (NaN on failure), status_out (NEGF_* codes,
 * NEGF_BAD_ITEM for an out-of-range system index, k index or block order
 * above max_order), iters_out (left lead's decimation sweeps); the last two
 * may be NULL.  blocks_per_sm: kernel variant (1 or 2, see
 * negf_batch_max_grid); grid: blocks (<= negf_batch_max_grid; <= 0 picks it).  The
 * launch (a counter reset and one kernel) can be captured in a CUDA graph once
 * a call with the same max_order and precision has run outside the capture.
 */
int negf_batch_transmission(const NegfBatchSystem* systems, int n_systems, int max_order, const int* item_system,
                            const int* item_k, const double* item_omega, int n_items, double tol, int maxiter,
                            int precision, int blocks_per_sm, int grid, double* t_out, int* status_out,
                            int* iters_out,
                            void* workspace, size_t workspace_bytes, void* stream);

/*
 * k average of an omega-major [n_omega][n_k] transmission table.
 * Replaces the mean in negfpy core/negf.py:360-397 (transmission_kavg).
 */
int negf_kavg_f64(const double* t, int n_omega, int n_k, double* t_mean, void* stream);

/*
 * Thermal conductance kappa(T_j) = (1/2pi) trapz(kB t_mean x^2 e^-x/(1-e^-x)^2, w)
 * with w = omega * omega_unit_rad_s and x = hbar w / (kB T_j).
 * Replaces negfpy workflows/ifc_bulk.py:408-438 (_thermal_conductance_from_spectrum).
 */
int negf_kappa_f64(const double* omega, const double* t_mean, int n_omega, const double* temperatures, int n_temps,
                   double omega_unit_rad_s, double* kappa_out, void* stream);

/*
 * k-space blocks of a force-constant model for n_k k-points at once:
 *   out[k] = diag(row_weight) (sum_t terms[t] exp(i (ky dy_t + kz dz_t)) + pinning I) diag(col_weight)
 * with real terms[n_terms][n][n], shifts[n_terms][2] = (dy, dz) and
 * kpoints[n_k][2] = (ky, kz); out is complex128 [n_k][n][n].  Replaces the
 * per-k phase sums and mass weighting of negfpy
 * models/material_kspace.py:99-128 (_sum_k_terms, _build_dynamical_blocks).
 * At most 256 terms.  Returns NEGF_EINVAL on a bad argument.
 */
int negf_kspace_blocks_f64(const double* terms, const double* shifts, int n_terms, const double* kpoints, int n_k,
                           int n, const double* row_weight, const double* col_weight, double pinning, double* out,
                           void* stream);

/*
 * k moments of an omega-major [n_omega][n_k] transmission table:
 * t_mean[w] = <T>_k, t2_mean[w] = <T^2>_k.  Replaces the per-omega moments
 * of negfpy workflows/ifc_bulk.py:1690-1784 (full counting statistics).
 */
int negf_kmoments_f64(const double* t, int n_omega, int n_k, double* t_mean, double* t2_mean, void* stream);

/*
 * First and second cumulants of the heat current from transmission moments
 * on a strictly increasing grid omega_rad_s (rad/s):
 *   c_out[0] = C1 (J/s) = (1/2pi) trapz(<T> (A_L - A_R), w),
 *   c_out[1] = C2 (J^2/s) = (1/2pi) trapz(<T> (B_L + B_R) + (<T> + <T^2>) (A_L - A_R)^2, w),
 * A = kB T x/expm1(x), B = (kB T)^2 x^2 e^x / expm1(x)^2, x = hbar w/(kB T).
 * Replaces negfpy core/fcs.py:48-150 (heat_current_cumulants_from_k_moments;
 * with t2_mean = T^2 also heat_current_cumulants_from_spectrum).
 */
int negf_fcs_cumulants_f64(const double* omega_rad_s, const double* t_mean, const double* t2_mean, int n_omega,
                           double temp_left, double temp_right, double* c_out, void* stream);

/*
 * Landauer heat current of n_spectra transmission rows t[b][n_omega] on one
 * strictly increasing grid omega_rad_s (rad/s):
 *   j[b] = (1/2pi) trapz((kB T_L phi(x_L) - kB T_R phi(x_R)) t[b], omega),
 *   phi(x) = x / expm1(x), x = hbar omega / (kB T), in W.
 * Replaces negfpy core/thermal_current.py:30-67 (heat_current_from_spectrum
 * and _spectral_bose_weight).  Temperatures must be positive.
 */
int negf_heat_current_f64(const double* omega_rad_s, const double* t, int n_omega, int n_spectra, double temp_left,
                          double temp_right, double* j_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* NEGF_B200_H */
