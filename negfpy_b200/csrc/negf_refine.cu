// Refined device solve: the RGF factorisation in FP32 on the tensor cores,
// corrected to FP64 accuracy by iterative refinement with FP64 residuals.
//
// Same contract as rgf_f64_global_kernel (negfpy core/negf.py:72-357): per
// point Sigma = V g V^H of both contacts from the FP64 surface GFs, the
// block-tridiagonal A = z - D - Sigma_L - Sigma_R, and
// T = Re Tr[Gamma_L G_{0,L-1} Gamma_R G_{0,L-1}^H].  negfpy solves A X = E_R
// for the right-contact block column X (core/negf.py:346-353); here:
//
//  1. FP32 left sweep (3 x TF32 products, FP32 Gauss-Jordan), keeping every
//     g_l = (z - D_l - C_{l-1}^H g_{l-1} C_{l-1} [- Sigma])^-1: the block LU
//     factors of A.
//  2. The last block column in FP32, X_{L-1} = g_{L-1},
//     X_i = g_i C_i X_{i+1}, widened to FP64.
//  3. Refinement steps: the residual R = E_R - A X in FP64 (three DMMA
//     products per layer), the correction A d = R with the FP32 factors
//     (forward y_i = g_i (R_i + C_{i-1}^H y_{i-1}), backward
//     d_i = y_i + g_i C_i d_{i+1}), X += d in FP64.  With
//     nu_k = max|d| / max|X| over all blocks after step k and the measured
//     contraction rho_k = nu_k / nu_{k-1}, the refinement stops at the first
//     k >= 2 with nu_k rho_k <= tol (the next correction, predicted from the
//     contraction, is below tol), or as soon as nu_k <= tol.  A step whose
//     correction did not shrink to half the previous one (rho_k > 1/2), or
//     no convergence within maxit steps, gives NEGF_REFINE_FAIL for the point
//     (the host solves those points again in FP64).
//  4. Gamma_L, Gamma_R and the trace in FP64 from X_0 = G_{0,L-1}.
#include "negf_common.cuh"
#include "negf_f64.h"
#include "negf_mixed.cuh"
#include "negf_tcprod.cuh"
#include "negf_tiles.cuh"

namespace negf {
namespace refine {

using glob::Acc;
using glob::kThreads;
using glob::kWarps;
using glob::Tile;
using glob::tc;
using glob::tile_mm;
using glob::tile_of;
using glob::tr;
using mixed::Acc32;
using mixed::GJS32;
using mixed::gj_invert32;
using mixed::load_pad32;
using mixed::tile_mm32;
using mixed::to_f;

// Workspace per block.  FP64: B0..B3 (self-energy scratch, then Sigma_L and
// Sigma_R padded, then the trace's scratch), the padded D_i, C_{i-1}, C_i,
// L slots of X, Sigma_L and Sigma_R (n x n).  FP32: L slots of g_l, L slots of
// y_i / d_i, and five NP x NP buffers (C, two temporaries, the inversion pair).
__host__ __device__ inline size_t ws64_elems(int np, int n, int L) {
  return (size_t)(7 + L) * np * np + 2 * (size_t)n * n;
}
__host__ __device__ inline size_t ws_bytes_per_block(int np, int n, int L) {
  return ws64_elems(np, n, L) * 16 + (size_t)(2 * L + 5) * np * np * 8;
}

__device__ __forceinline__ void widen_pad(double2* dst, const float2* src, int n, int NP) {
  for (long long e = threadIdx.x; e < (long long)NP * NP; e += kThreads) {
    const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
    const float2 v = src[e];
    dst[e] = (r < n && c < n) ? make_double2((double)v.x, (double)v.y) : make_double2(0.0, 0.0);
  }
}
__device__ __forceinline__ void copy32(float2* dst, const float2* src, int NP) {
  for (long long e = threadIdx.x; e < (long long)NP * NP; e += kThreads) dst[e] = src[e];
}
// n x n FP64 (row stride n) -> padded NP x NP FP64 with zeros outside.
__device__ __forceinline__ void pad64(double2* dst, const double2* src, int n, int NP) {
  glob::load_pad(dst, src, n, n, NP, 0.0);
}

// dst = op(A) op(B) for padded NP x NP FP32 matrices: on tcgen05 (TC; the
// block's context *tcx) or on 3 x TF32 mma.sync tiles (contraction over the
// kch chunks of the logical order).  Ends with the block synchronised;
// false if a tcgen05 completion wait ran out.
template <bool TC, bool AC, bool BC>
__device__ bool prod32(float2* dst, const float2* A, const float2* B, int NP, int kch, tc::Ctx* tcx) {
  if constexpr (TC) {
    return tc::cprod<AC, BC>(dst, A, B, NP, *tcx);
  } else {
    const int np16 = NP >> 4, ntiles = np16 * np16;
    for (int tt = threadIdx.x >> 5; tt < ntiles; tt += kWarps) {
      const Tile T = tile_of(tt, np16);
      Acc32 c1;
      tile_mm32<AC, BC>(c1, A, B, NP, kch, T);
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) dst[(long long)tr(T, qq) * NP + tc(T, j, qq)] = c1.get(j, qq);
    }
    __syncthreads();
    return true;
  }
}

template <bool TC>
static __device__ int refine_point(const glob::RgfPoint& q, int NP, unsigned char* blk, const GJS32& sh,
                                   double* red, double tol, int maxit, double* t, int* steps, tc::Ctx* tcx) {
  const int n = q.n, L = q.L, tid = threadIdx.x, warp = tid >> 5;
  const int np16 = NP >> 4, ntiles = np16 * np16, kch = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  double2* d64 = reinterpret_cast<double2*>(blk);
  double2 *B0 = d64, *B1 = d64 + M2, *B2 = d64 + 2 * M2, *B3 = d64 + 3 * M2;
  double2 *Dp = d64 + 4 * M2, *Cm = d64 + 5 * M2, *Cn = d64 + 6 * M2;
  double2* X64 = d64 + 7 * M2;
  double2* sigL = X64 + (long long)L * M2;
  double2* sigR = sigL + (long long)n * n;
  float2* f32 = reinterpret_cast<float2*>(blk + ws64_elems(NP, n, L) * 16);
  float2* gs = f32;
  float2* ys = gs + (long long)L * M2;
  float2 *pc = ys + (long long)L * M2, *tA = pc + M2, *tB = tA + M2, *bM = tB + M2, *bX = bM + M2;
  const double2 z = q.z;
  auto Dl = [&](int l) { return q.D + (long long)l * q.d_ls; };
  auto Cl = [&](int l) { return q.C + (long long)l * q.c_ls; };
  *steps = 0;

  glob::self_energies(q, NP, B0, B1, B2, sigL, sigR);
  // 1. FP32 left sweep; g_l kept in slot l.
  int status = kOk;
  for (int l = 0; l < L && status == kOk; ++l) {
    if (l > 0) {
      load_pad32(pc, Cl(l - 1), n, NP);
      __syncthreads();
      bool ok = prod32<TC, false, false>(tA, gs + (l - 1) * M2, pc, NP, kch, tcx);  // g_{l-1} C_{l-1}
      ok = prod32<TC, true, false>(bX, pc, tA, NP, kch, tcx) && ok;                 // C^H g C
      if (!ok) {
        status = kNonFinite;
        break;
      }
    }
    // M_l = z - D_l [- Sigma_L] [- Sigma_R] - C^H g C; the FP64 terms are
    // combined in FP64 before the rounding.
    const double2* D = Dl(l);
    for (long long e = tid; e < M2; e += kThreads) {
      const int r = (int)(e / NP), cc = (int)(e - (long long)r * NP);
      float2 v;
      if (r < n && cc < n) {
        double2 w = cneg(D[r * n + cc]);
        if (l == 0) w = csub(w, sigL[r * n + cc]);
        if (l == L - 1) w = csub(w, sigR[r * n + cc]);
        if (r == cc) w = cadd(w, z);
        const float2 x = l > 0 ? bX[e] : make_float2(0.f, 0.f);
        v = make_float2((float)(w.x - (double)x.x), (float)(w.y - (double)x.y));
      } else {
        v = make_float2(r == cc ? 1.f : 0.f, 0.f);
      }
      bM[e] = v;
    }
    __syncthreads();
    float2* inv = nullptr;
    status = gj_invert32(bM, bX, n, NP, sh, &inv);
    if (status != kOk) break;
    copy32(gs + l * M2, inv, NP);
    __syncthreads();
  }
  if (status != kOk) {
    __syncthreads();
    *t = 0.0;
    return status;
  }
  // 2. Last block column in FP32, widened into X64.
  copy32(tA, gs + (L - 1) * M2, NP);
  widen_pad(X64 + (L - 1) * M2, gs + (L - 1) * M2, n, NP);
  __syncthreads();
  for (int i = L - 2; i >= 0 && status == kOk; --i) {
    load_pad32(pc, Cl(i), n, NP);
    __syncthreads();
    bool ok = prod32<TC, false, false>(tB, pc, tA, NP, kch, tcx);           // C_i X_{i+1}
    ok = prod32<TC, false, false>(tA, gs + i * M2, tB, NP, kch, tcx) && ok;  // X_i = g_i C_i X_{i+1}
    if (!ok) status = kNonFinite;
    widen_pad(X64 + i * M2, tA, n, NP);
    __syncthreads();
  }
  // Sigma_L and Sigma_R padded for the residual products.
  pad64(B0, sigL, n, NP);
  pad64(B1, sigR, n, NP);
  __syncthreads();

  // 3. Refinement.
  double nu_prev = 0.0;
  bool done = false;
  for (int it = 1; it <= maxit && !done && status == kOk; ++it) {
    *steps = it;
    // forward: R_i in FP64, t_i = R_i + C_{i-1}^H y_{i-1}, y_i = g_i t_i
    for (int i = 0; i < L && status == kOk; ++i) {
      pad64(Dp, Dl(i), n, NP);
      if (i > 0) {
        pad64(Cm, Cl(i - 1), n, NP);
        load_pad32(pc, Cl(i - 1), n, NP);
      }
      if (i < L - 1) pad64(Cn, Cl(i), n, NP);
      __syncthreads();
      if (i > 0 && !prod32<TC, true, false>(bM, pc, ys + (i - 1) * M2, NP, kch, tcx)) {
        status = kNonFinite;
        break;
      }
      const double2* Xi = X64 + i * M2;
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc a;  // D_i X_i + C_{i-1}^H X_{i-1} + C_i X_{i+1} + Sigma X_i at the ends
        tile_mm<false, false>(a, Dp, NP, Xi, NP, kch, T);
        if (i > 0) tile_mm<true, false, true>(a, Cm, NP, Xi - M2, NP, kch, T);
        if (i < L - 1) tile_mm<false, false, true>(a, Cn, NP, Xi + M2, NP, kch, T);
        if (i == 0) tile_mm<false, false, true>(a, B0, NP, Xi, NP, kch, T);
        if (i == L - 1) tile_mm<false, false, true>(a, B1, NP, Xi, NP, kch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int qq = 0; qq < 4; ++qq) {
            const int r = tr(T, qq), cc = tc(T, j, qq);
            const long long e = (long long)r * NP + cc;
            float2 v = make_float2(0.f, 0.f);
            if (r < n && cc < n) {
              // R = E - (z X - D X - C^H X - C X - Sigma X)
              double2 rv = csub(a.get(j, qq), cmul(z, Xi[e]));
              if (i == L - 1 && r == cc) rv.x += 1.0;
              const float2 cy = i > 0 ? bM[e] : make_float2(0.f, 0.f);
              v = make_float2((float)rv.x + cy.x, (float)rv.y + cy.y);
            }
            tA[e] = v;
          }
      }
      __syncthreads();
      if (!prod32<TC, false, false>(ys + i * M2, gs + i * M2, tA, NP, kch, tcx)) status = kNonFinite;  // y_i
    }
    if (status != kOk) break;
    // backward: d_{L-1} = y_{L-1}, d_i = y_i + g_i C_i d_{i+1}; X += d
    double dmax = 0.0, xmax = 0.0;
    for (int i = L - 1; i >= 0; --i) {
      float2* yi = ys + i * M2;
      double2* Xi = X64 + i * M2;
      if (i < L - 1) {
        load_pad32(pc, Cl(i), n, NP);
        __syncthreads();
        bool ok = prod32<TC, false, false>(tB, pc, yi + M2, NP, kch, tcx);        // C_i d_{i+1}
        ok = prod32<TC, false, false>(bM, gs + i * M2, tB, NP, kch, tcx) && ok;  // g_i C_i d_{i+1}
        if (!ok) {
          status = kNonFinite;
          break;
        }
      }
      for (long long e = tid; e < M2; e += kThreads) {
        const int r = (int)(e / NP), cc = (int)(e - (long long)r * NP);
        const float2 y = yi[e];
        const float2 c1 = i < L - 1 ? bM[e] : make_float2(0.f, 0.f);
        const float2 d = make_float2(__fadd_rn(y.x, c1.x), __fadd_rn(y.y, c1.y));
        yi[e] = d;
        if (r < n && cc < n) {
          const double2 x = cadd(Xi[e], make_double2((double)d.x, (double)d.y));
          Xi[e] = x;
          dmax = fmax(dmax, fmax(fabs((double)d.x), fabs((double)d.y)));
          xmax = fmax(xmax, fmax(fabs(x.x), fabs(x.y)));
        }
      }
      __syncthreads();
    }
    if (status != kOk) break;
    int bad = !(isfinite(dmax) && isfinite(xmax));
    if (block_any(bad)) {
      status = kNonFinite;
      break;
    }
    dmax = block_max(dmax, red);
    xmax = block_max(xmax, red);
    const double nu = xmax > 0.0 ? dmax / xmax : 0.0;
    if (nu <= tol) {
      done = true;
    } else if (it >= 2) {
      const double rho = nu / nu_prev;
      if (rho > 0.5) {
        status = kRefineFail;  // the correction stopped shrinking
        break;
      }
      if (nu * rho <= tol) done = true;
    }
    nu_prev = nu;
  }
  if (status == kOk && !done) status = kRefineFail;
  // 4. Gamma and trace in FP64 from X_0 = G_{0,L-1}.
  double tval = 0.0;
  if (status == kOk) {
    tval = glob::trace_t(n, NP, sigL, sigR, X64, B0, B1, B3, red);
    if (!isfinite(tval)) status = kNonFinite;
  } else {
    __syncthreads();
  }
  *t = tval;
  return status;
}

// Dynamic shared memory: [tcgen05 stage and mbarrier (TC only) | GJ panel,
// pivot bookkeeping | reduction scratch].  With TC at least 80 KB, so that at
// most two blocks share an SM and their TMEM (2 x 256 columns) always fits.
__host__ __device__ inline size_t tc_bytes(int np) { return ((tc::stage_bytes(np) + 16 + 127) / 128) * 128; }
template <bool TC>
size_t smem_bytes(int np) {
  const size_t base = ((mixed::gjs32_bytes(np) + 15) / 16) * 16 + 40 * 8;
  if (!TC) return base;
  const size_t need = tc_bytes(np) + base;
  return need > 80 * 1024 ? need : 80 * 1024;
}

template <bool TC>
__global__ void __launch_bounds__(kThreads, 2) rgf_refine_kernel(RgfArgs a, int NP, unsigned char* ws, double tol,
                                                                 int maxit, int* steps_out) {
  extern __shared__ __align__(128) unsigned char smraw[];
  unsigned char* gj = smraw + (TC ? tc_bytes(NP) : 0);
  const GJS32 sh = mixed::carve32(gj, NP);
  double* red = reinterpret_cast<double*>(gj + ((mixed::gjs32_bytes(NP) + 15) / 16) * 16);
  __shared__ int s_point;
  __shared__ uint32_t s_tmem;
  __shared__ int s_tcerr;
  const int n = a.n, tid = threadIdx.x;
  unsigned char* blk = ws + (long long)blockIdx.x * ws_bytes_per_block(NP, n, a.L);
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
        if (steps_out) steps_out[p] = 0;
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
    int steps = 0;
    const int status = refine_point<TC>(q, NP, blk, sh, red, tol, maxit, &tval, &steps, &tcx);
    if (tid == 0) {
      a.T_out[p] = (status == kOk) ? tval : __longlong_as_double(0x7ff8000000000000ULL);
      if (a.status_out) a.status_out[p] = status;
      if (steps_out) steps_out[p] = steps;
    }
    __syncthreads();
  }
  if constexpr (TC) tc::teardown(tcx);
}

}  // namespace refine

bool refine_use_tc(int np) { return mixed::use_tc(np); }

int rgf_refine_grid(int np) {
  const bool tcp = refine_use_tc(np);
  const size_t sm = tcp ? refine::smem_bytes<true>(np) : refine::smem_bytes<false>(np);
  auto kernel = tcp ? refine::rgf_refine_kernel<true> : refine::rgf_refine_kernel<false>;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return -3;
  int nb = 0, dev = 0, nsm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, refine::kThreads, sm) != cudaSuccess || nb <= 0)
    return -3;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (nb > 2) nb = 2;  // the L-slot workspace grows with the grid; two blocks' TMEM per SM
  return nb * nsm;
}
size_t rgf_refine_ws_bytes(int np, int n, int L, int grid) {
  return (size_t)grid * refine::ws_bytes_per_block(np, n, L);
}
int rgf_refine_launch(const RgfArgs& a, int np, int grid, void* ws, double tol, int maxit, int* steps_out,
                      cudaStream_t st) {
  if (a.batch <= 0) return 0;
  if (refine_use_tc(np)) {
    refine::rgf_refine_kernel<true><<<grid, refine::kThreads, refine::smem_bytes<true>(np), st>>>(
        a, np, static_cast<unsigned char*>(ws), tol, maxit, steps_out);
  } else {
    refine::rgf_refine_kernel<false><<<grid, refine::kThreads, refine::smem_bytes<false>(np), st>>>(
        a, np, static_cast<unsigned char*>(ws), tol, maxit, steps_out);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace negf
