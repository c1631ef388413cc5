// FP64 kernels for block orders 49..256 (padded to NP, a multiple of 16).
//
// One point's matrices do not fit one SM's shared memory beyond n = 48, so
// here they live in a per-block workspace in global memory (mostly L2
// resident) and the blocks are persistent: each takes points from an atomic
// counter.  The decimation and sweep kernels are register-capped for two
// resident blocks per SM (128 registers a thread, a few hundred bytes of
// spill), so one point's latency-bound pivot steps overlap another's
// products: 1.22x (decimation) and 1.33x (sweep) faster at n = 96 than one
// uncapped block per SM.
// Row-major, row stride NP, no swizzle (global accesses of a warp fragment are
// 16-byte loads from at most 8 rows).
//
//   sr_f64_global_kernel   Sancho-Rubio decimation, same recurrence, stopping
//                          rule and outputs as sr_f64_kernel (negfpy
//                          core/surface_gf.py:18-81).
//   rgf_f64_global_kernel  Sigma, left-connected RGF sweep and trace, as
//                          rgf_f64_kernel (negfpy core/negf.py:72-357).
//
// Products: each warp walks 16 x 16 output tiles (two m16n8 DMMA tiles) in
// a strided loop; complex = four real mma.sync m16n8k8 f64.  Inversion:
// blocked Gauss-Jordan, 8-column panels factored by the whole block in
// shared memory with the division-free, look-ahead rule of the
// shared-memory kernels, the rank-8 update of the whole matrix between two
// global buffers on DMMA, and a final column gather.
#include <cstdio>

#include "negf_common.cuh"
#include "negf_f64.h"
#include "negf_point.cuh"
#include "negf_tiles.cuh"

namespace negf {
namespace glob {

// ------------------------------------------------------------ Sancho-Rubio --
// Workspace per block: 7 NP x NP buffers (alpha, beta, eps, eps_s, three free).
__global__ void __launch_bounds__(kThreads, 2) sr_f64_global_kernel(SrArgs a, int NP, double2* ws, unsigned* counter) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const GJS sh = carve(smraw, NP);
  double* red = reinterpret_cast<double*>(smraw + ((gjs_bytes(NP) + 15) / 16) * 16);
  __shared__ int s_point;
  const int n = a.n, tid = threadIdx.x;
  const long long M2 = (long long)NP * NP;
  double2* base = ws + (long long)blockIdx.x * 7 * M2;

  for (;;) {
    if (tid == 0) s_point = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int p = s_point;
    __syncthreads();
    if (p >= a.batch) break;
    const long long kset = a.kidx ? (long long)a.kidx[p] : 0;
    const double2* h00 = a.h00 + kset * a.lead_stride;
    const double2* h01 = a.h01 + kset * a.lead_stride;
    const double2* h10 = a.h10 ? a.h10 + kset * a.lead_stride : nullptr;
    const double w = a.omega[p];
    int it = 0;
    double2* pg = nullptr;
    const int status = sr_point(n, NP, h00, h01, h10, z_of(w, a.eta[p]), a.tol, a.maxiter, base, sh, red, &it, &pg);
    if (status == kOk) {
      if (a.g_out) {
        double2* go = a.g_out + (long long)p * n * n;
        for (int e = tid; e < n * n; e += kThreads) {
          const int r = e / n, c = e - r * n;
          go[e] = pg[(long long)r * NP + c];
        }
      }
      if (a.dos_out) {
        double t = 0.0;
        for (int j = tid; j < n; j += kThreads) t += -2.0 * pg[(long long)j * NP + j].y;
        t = block_sum(t, red);
        if (tid == 0) a.dos_out[p] = (w / 3.141592653589793238462643383279502884) * t;
      }
    } else if (a.dos_out && tid == 0) {
      a.dos_out[p] = __longlong_as_double(0x7ff8000000000000ULL);
    }
    if (tid == 0) {
      if (a.iters_out) a.iters_out[p] = it;
      if (a.status_out) a.status_out[p] = status;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- RGF sweep --
// Workspace per block: 6 NP x NP buffers (g, second inversion buffer, W, U,
// G0, scratch) and Sigma_L, Sigma_R (n x n each).
__global__ void __launch_bounds__(kThreads, 2) rgf_f64_global_kernel(RgfArgs a, int NP, double2* ws) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const GJS sh = carve(smraw, NP);
  double* red = reinterpret_cast<double*>(smraw + ((gjs_bytes(NP) + 15) / 16) * 16);
  __shared__ int s_point;
  const int n = a.n, tid = threadIdx.x;
  const long long M2 = (long long)NP * NP;
  double2* base = ws + (long long)blockIdx.x * (6 * M2 + 2LL * n * n);

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
    RgfPoint q;
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
    q.z = z_of(a.omega[p], a.eta_dev[p]);
    double tval = 0.0;
    const int status = rgf_point_f64(q, NP, base, sh, red, &tval);
    if (tid == 0) {
      a.T_out[p] = (status == kOk) ? tval : __longlong_as_double(0x7ff8000000000000ULL);
      if (a.status_out) a.status_out[p] = status;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------- adjoint (gradient) --
// Whole-matrix helpers over the (NP/16)^2 tiles of a block (each ends with a
// barrier).
template <bool AC, bool BC>
__device__ void gemm_to(double2* dst, const double2* A, const double2* B, int NP, int kch) {
  const int warp = threadIdx.x >> 5, np16 = NP >> 4, nt = np16 * np16;
  for (int tt = warp; tt < nt; tt += kWarps) {
    const Tile T = tile_of(tt, np16);
    Acc c;
    tile_mm<AC, BC>(c, A, NP, B, NP, kch, T);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) dst[(long long)tr(T, q) * NP + tc(T, j, q)] = c.get(j, q);
  }
  __syncthreads();
}
// dst = z - D - op(A) op(B) [- S1] [- S2] on the leading n x n block, identity
// padding; A == nullptr drops the product.
template <bool AC, bool BC>
__device__ void form_m(double2* dst, const double2* A, const double2* B, const double2* __restrict__ D,
                       const double2* S1, const double2* S2, double2 z, int n, int NP, int kch) {
  const int warp = threadIdx.x >> 5, np16 = NP >> 4, nt = np16 * np16;
  for (int tt = warp; tt < nt; tt += kWarps) {
    const Tile T = tile_of(tt, np16);
    Acc c;
    if (A) tile_mm<AC, BC>(c, A, NP, B, NP, kch, T);
    else c.zero();
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = tr(T, q), cc = tc(T, j, q);
        double2 v;
        if (r < n && cc < n) {
          v = csub(cneg(D[r * n + cc]), c.get(j, q));
          if (S1) v = csub(v, S1[r * n + cc]);
          if (S2) v = csub(v, S2[r * n + cc]);
          if (r == cc) v = cadd(v, z);
        } else {
          v = make_double2(r == cc ? 1.0 : 0.0, 0.0);
        }
        dst[(long long)r * NP + cc] = v;
      }
  }
  __syncthreads();
}
__device__ void copy_mat(double2* dst, const double2* src, int NP) {
  for (long long e = threadIdx.x; e < (long long)NP * NP; e += kThreads) dst[e] = src[e];
  __syncthreads();
}
// Inverse of the matrix formed in `slot`, left in `slot` (Y is scratch).
__device__ int invert_into(double2* slot, double2* Y, int n, int NP, const GJS& sh) {
  double2* out = nullptr;
  const int st = gj_invert_global(slot, Y, n, NP, sh, &out);
  if (st == kOk && out != slot) copy_mat(slot, out, NP);
  return st;
}
__device__ __forceinline__ void atomic_cadd(double2* dst, double2 v) {
  atomicAdd(&dst->x, v.x);
  atomicAdd(&dst->y, v.y);
}
// A point's contribution to a gradient block: added atomically into the
// shared per-k block, or stored into the point's own block (per-point mode,
// which the host then sums in a fixed order for a reproducible result).
__device__ __forceinline__ void grad_put(double2* dst, double2 v, bool own) {
  if (own) *dst = v;
  else atomic_cadd(dst, v);
}

// Per point: T and the weighted adjoint blocks of dT/dD.  With G = A^-1 for
// A = z - D - Sigma_L - Sigma_R, Y = Gamma_R G_{0,L-1}^H Gamma_L and
// X_{ji} = G_{j,L-1} Y G_{0,i},
//     dT = 2 Re sum_ij Tr[dD_ij X_ji],
// so a change dD_i of onsite block i contributes 2 Re Tr[dD_i X_ii] and a
// change dC_i of the coupling between layers i and i+1 (with dC_i^H below the
// diagonal) contributes 2 Re Tr[dC_i (X_{i+1,i} + X_{i,i+1}^H)].  The kernel
// adds weight[p] X_ii into grad_d[k][i] and weight[p] (X_{i+1,i} + X_{i,i+1}^H)
// into grad_c[k][i].  Nothing is kept from the forward pass: the left sweep
// (g^L), the last block column G_{j,L-1} (backward recursion), the right sweep
// (g^R) and the first block row G_{0,i} are recomputed here, per point.
__global__ void __launch_bounds__(kThreads, 2) rgf_grad_f64_kernel(GradArgs ga, int NP, double2* ws) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const GJS sh = carve(smraw, NP);
  double* red = reinterpret_cast<double*>(smraw + ((gjs_bytes(NP) + 15) / 16) * 16);
  __shared__ int s_point;
  const RgfArgs& a = ga.r;
  const int n = a.n, L = a.L, tid = threadIdx.x;
  const int kch = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  double2* base = ws + (long long)blockIdx.x * ((14 + 2LL * L) * M2 + 2LL * n * n);
  double2* B[14];
  for (int i = 0; i < 14; ++i) B[i] = base + i * M2;
  double2* gl = base + 14 * M2;             // L slots: g^L_j, then G_{j,L-1}
  double2* gr = gl + (long long)L * M2;     // L slots: g^R_i
  double2* sigL = gr + (long long)L * M2;
  double2* sigR = sigL + (long long)n * n;
  double2 *Cb = B[0], *W = B[1], *Mb = B[2], *Xs = B[3], *GL = B[4], *GR = B[5], *Y = B[6];
  double2 *Ap = B[7], *Ac = B[8], *G0p = B[9], *G0c = B[10], *Xa = B[11], *Xb = B[12], *Tt = B[13];

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
    const double2 z = z_of(a.omega[p], a.eta_dev[p]);
    const double2* D = a.D + k * a.d_ks;
    const double2* C = a.C + k * a.c_ks;
    const double wgt = ga.weight[p];
    const bool own = ga.per_point != 0;
    const long long slot = own ? (long long)p : k;
    double2* gdk = ga.grad_d + slot * (long long)L * n * n;
    double2* gck = ga.grad_c + slot * (long long)(L > 1 ? L - 1 : 1) * n * n;
    auto Dl = [&](int l) { return D + (long long)l * a.d_ls; };
    auto load_c = [&](int l) {
      load_pad(Cb, C + (long long)l * a.c_ls, n, n, NP, 0.0);
      __syncthreads();
    };

    // Sigma and Gamma of both contacts.
    for (int side = 0; side < 2; ++side) {
      const int nl = side ? a.nr : a.nl;
      const int lch = (nl + 7) >> 3;
      const double2* V = side ? a.VR + k * a.vr_ks : a.VL + k * a.vl_ks;
      const double2* g = side ? a.gR + (long long)p * a.gr_ps : a.gL + (long long)p * a.gl_ps;
      double2* S = side ? sigR : sigL;
      load_pad(W, V, n, nl, NP, 0.0);
      load_pad(Xs, g, nl, nl, NP, 0.0);
      __syncthreads();
      gemm_to<false, false>(Tt, W, Xs, NP, lch);
      gemm_to<false, true>(Mb, Tt, W, NP, lch);
      for (long long e = tid; e < M2; e += kThreads) {
        const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
        if (r < n && c < n) S[r * n + c] = Mb[e];
      }
      __syncthreads();
    }
    for (long long e = tid; e < M2; e += kThreads) {
      const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
      double2 gl_ = make_double2(0.0, 0.0), gr_ = gl_;
      if (r < n && c < n) {
        double2 d = csub(sigL[r * n + c], cconj(sigL[c * n + r]));
        gl_ = make_double2(-d.y, d.x);
        d = csub(sigR[r * n + c], cconj(sigR[c * n + r]));
        gr_ = make_double2(-d.y, d.x);
      }
      GL[e] = gl_;
      GR[e] = gr_;
    }
    __syncthreads();

    int status = kOk;
    // 1. left sweep: gl[l] = g^L_l
    form_m<false, false>(gl, nullptr, nullptr, Dl(0), sigL, L == 1 ? sigR : nullptr, z, n, NP, kch);
    status = invert_into(gl, Xs, n, NP, sh);
    for (int l = 1; l < L && status == kOk; ++l) {
      load_c(l - 1);
      gemm_to<false, false>(W, gl + (l - 1) * M2, Cb, NP, kch);
      form_m<true, false>(gl + l * M2, Cb, W, Dl(l), l == L - 1 ? sigR : nullptr, nullptr, z, n, NP, kch);
      status = invert_into(gl + l * M2, Xs, n, NP, sh);
    }
    // 2. last block column: G_{L-1,L-1} = g^L_{L-1}, G_{j,L-1} = g^L_j C_j G_{j+1,L-1}
    for (int j = L - 2; j >= 0 && status == kOk; --j) {
      load_c(j);
      gemm_to<false, false>(W, Cb, gl + (j + 1) * M2, NP, kch);
      gemm_to<false, false>(Tt, gl + j * M2, W, NP, kch);
      copy_mat(gl + j * M2, Tt, NP);
    }
    double tval = 0.0;
    if (status == kOk) {
      // T = Re Tr[Gamma_L G Gamma_R G^H], G = G_{0,L-1};  Y = Gamma_R G^H Gamma_L
      gemm_to<false, false>(Tt, GL, gl, NP, kch);
      gemm_to<false, false>(W, Tt, GR, NP, kch);
      double t = 0.0;
      for (long long e = tid; e < M2; e += kThreads) t += W[e].x * gl[e].x + W[e].y * gl[e].y;
      tval = block_sum(t, red);
      if (!isfinite(tval)) status = kNonFinite;
      gemm_to<true, false>(Tt, gl, GL, NP, kch);
      gemm_to<false, false>(Y, GR, Tt, NP, kch);
    }
    // 3. right sweep: gr[i] = g^R_i, then G_{0,0}
    if (status == kOk) {
      form_m<false, false>(gr + (L - 1) * M2, nullptr, nullptr, Dl(L - 1), sigR, L == 1 ? sigL : nullptr, z, n, NP,
                           kch);
      status = invert_into(gr + (L - 1) * M2, Xs, n, NP, sh);
      for (int i = L - 2; i >= 1 && status == kOk; --i) {
        load_c(i);
        gemm_to<false, false>(W, Cb, gr + (i + 1) * M2, NP, kch);
        form_m<false, true>(gr + i * M2, W, Cb, Dl(i), nullptr, nullptr, z, n, NP, kch);
        status = invert_into(gr + i * M2, Xs, n, NP, sh);
      }
      if (status == kOk) {
        if (L == 1) {
          copy_mat(G0c, gr, NP);
        } else {
          load_c(0);
          gemm_to<false, false>(W, Cb, gr + M2, NP, kch);
          form_m<false, true>(G0c, W, Cb, Dl(0), sigL, nullptr, z, n, NP, kch);
          status = invert_into(G0c, Xs, n, NP, sh);
        }
      }
    }
    // Contact terms of dT/dSigma: Sigma_L enters A_00 (like D_00) and Gamma_L,
    // so dT/dSigma_L = X_00 + i G Gamma_R G^H; likewise dT/dSigma_R =
    // X_{L-1,L-1} + i G^H Gamma_L G, with G = G_{0,L-1} (slot 0 of gl).
    const bool want_l = ga.sig_adj_l != nullptr, want_r = ga.sig_adj_r != nullptr;
    if (status == kOk && want_l) {
      gemm_to<false, false>(W, gl, GR, NP, kch);
      gemm_to<false, true>(Mb, W, gl, NP, kch);
    }
    if (status == kOk && want_r) {
      gemm_to<true, false>(W, gl, GL, NP, kch);
      gemm_to<false, false>(Xs, W, gl, NP, kch);
    }
    // 4. first block row and the adjoint blocks
    for (int i = 0; i < L && status == kOk; ++i) {
      gemm_to<false, false>(Ac, gl + i * M2, Y, NP, kch);
      gemm_to<false, false>(Xa, Ac, G0c, NP, kch);
      for (long long e = tid; e < M2; e += kThreads) {
        const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
        if (r < n && c < n) {
          const double2 v = Xa[e];
          grad_put(gdk + (long long)i * n * n + r * n + c, make_double2(wgt * v.x, wgt * v.y), own);
          if (i == 0 && want_l) {
            const double2 zt = Mb[e];
            ga.sig_adj_l[(long long)p * n * n + r * n + c] = make_double2(wgt * (v.x - zt.y), wgt * (v.y + zt.x));
          }
          if (i == L - 1 && want_r) {
            const double2 zt = Xs[e];
            ga.sig_adj_r[(long long)p * n * n + r * n + c] = make_double2(wgt * (v.x - zt.y), wgt * (v.y + zt.x));
          }
        }
      }
      __syncthreads();  // Xa is rewritten next
      if (i >= 1) {
        gemm_to<false, false>(Xa, Ac, G0p, NP, kch);   // X_{i,i-1}
        gemm_to<false, false>(Xb, Ap, G0c, NP, kch);   // X_{i-1,i}
        for (long long e = tid; e < M2; e += kThreads) {
          const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
          if (r < n && c < n) {
            const double2 v = cadd(Xa[e], cconj(Xb[(long long)c * NP + r]));
            grad_put(gck + (long long)(i - 1) * n * n + r * n + c, make_double2(wgt * v.x, wgt * v.y), own);
          }
        }
      }
      if (i + 1 < L) {
        load_c(i);
        gemm_to<false, false>(Tt, G0c, Cb, NP, kch);
        gemm_to<false, false>(G0p, Tt, gr + (i + 1) * M2, NP, kch);  // G_{0,i+1} into the spare buffer
        double2* t = G0p;
        G0p = G0c;
        G0c = t;
        t = Ap;
        Ap = Ac;
        Ac = t;
      }
    }
    __syncthreads();
    if (tid == 0) {
      a.T_out[p] = (status == kOk) ? tval : __longlong_as_double(0x7ff8000000000000ULL);
      if (a.status_out) a.status_out[p] = status;
    }
    __syncthreads();
  }
}

// ------------------------------------------------ adjoint of the surface GF --
// dst += op(A) op(B) (each thread updates only the elements of its own tiles).
template <bool AC, bool BC>
__device__ void gemm_add(double2* dst, const double2* A, const double2* B, int NP, int kch) {
  const int warp = threadIdx.x >> 5, np16 = NP >> 4, nt = np16 * np16;
  for (int tt = warp; tt < nt; tt += kWarps) {
    const Tile T = tile_of(tt, np16);
    Acc c;
    tile_mm<AC, BC>(c, A, NP, B, NP, kch, T);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double2* d = dst + (long long)tr(T, q) * NP + tc(T, j, q);
        *d = cadd(*d, c.get(j, q));
      }
  }
  __syncthreads();
}

// Per point, with the surface GF g of the lead (negfpy core/surface_gf.py:18-81
// computes it by decimation) and the weighted adjoint X of Sigma = V g V^H
// from rgf_grad_f64_kernel (dT = 2 Re Tr[dSigma X]):
//
//   gbar = V^H X V,   Vbar = g V^H X + g^H V^H X^H            (dT = 2 Re Tr[dV Vbar])
//
// g solves g = (z - H00 - H01 g H10)^-1, so with P = g H01 and Q = H10 g,
//   dg - P dg Q = g (dH00 + dH01 g H10 + H01 g dH10) g,
// and Tr[dg gbar] = Tr[(dH00 + dH01 g H10 + H01 g dH10) g Lam g] where Lam
// solves the transposed equation Lam - Q Lam P = gbar.  Lam = sum_k Q^k gbar P^k
// is summed by doubling (Smith's method): Lam += A Lam B, A <- A^2, B <- B^2
// from A = Q, B = P, until max(max|A|, max|B|) < tol; no inverse is needed and
// nothing is differentiated through the decimation sweeps.  Then
//   H00bar = g Lam g,  H01bar = g H10 H00bar,  H10bar = H00bar H01 g,
// added into the per-k accumulators (with H10 = H01^H, H10bar^H is added to
// H01bar instead).  Status: kMaxIter if the doubling does not converge within
// maxiter, kNonFinite on inf/nan.
__global__ void __launch_bounds__(kThreads, 2) sgf_adjoint_f64_kernel(SgfAdjArgs sa, int NP, double2* ws) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double* red = reinterpret_cast<double*>(smraw + ((gjs_bytes(NP) + 15) / 16) * 16);
  __shared__ int s_point;
  const int nl = sa.nl, n = sa.n, tid = threadIdx.x;
  const int kl = (nl + 7) >> 3, kd = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  double2* base = ws + (long long)blockIdx.x * 15 * M2;
  double2 *Vb = base, *Xb = base + M2, *Gb = base + 2 * M2, *T1 = base + 3 * M2, *T2 = base + 4 * M2;
  double2 *Gbar = base + 5 * M2, *Pk = base + 6 * M2, *Aq = base + 7 * M2, *Bp = base + 8 * M2;
  double2 *Aq2 = base + 9 * M2, *Bp2 = base + 10 * M2, *Lam = base + 11 * M2, *Tt = base + 12 * M2;
  double2 *H01b = base + 13 * M2, *H10b = base + 14 * M2;

  for (;;) {
    if (tid == 0) s_point = (int)atomicAdd(sa.counter, 1u);
    __syncthreads();
    const int p = s_point;
    __syncthreads();
    if (p >= sa.batch) break;
    const int lst = sa.lead_status ? sa.lead_status[p] : 0;
    if (lst != kOk) {
      if (tid == 0) {
        if (sa.status_out) sa.status_out[p] = lst;
        if (sa.iters_out) sa.iters_out[p] = 0;
      }
      continue;
    }
    const long long k = sa.kidx ? (long long)sa.kidx[p] : 0;
    const double2* h01 = sa.h01 + k * sa.lead_stride;
    const double2* h10 = sa.h10 ? sa.h10 + k * sa.lead_stride : nullptr;
    load_pad(Vb, sa.V + k * sa.v_ks, n, nl, NP, 0.0);
    load_pad(Xb, sa.xs + (long long)p * n * n, n, n, NP, 0.0);
    load_pad(Gb, sa.g + (long long)p * sa.g_ps, nl, nl, NP, 0.0);
    load_pad(H01b, h01, nl, nl, NP, 0.0);
    if (h10) load_pad(H10b, h10, nl, nl, NP, 0.0);
    __syncthreads();
    // gbar and Vbar
    gemm_to<false, false>(T1, Xb, Vb, NP, kd);     // X V          (n x nl)
    gemm_to<true, false>(Gbar, Vb, T1, NP, kd);    // V^H X V      (nl x nl)
    gemm_to<true, false>(T2, Vb, Xb, NP, kd);      // V^H X        (nl x n)
    gemm_to<false, false>(Aq, Gb, T2, NP, kl);     // g V^H X      (nl x n)
    gemm_to<false, false>(Bp, T1, Gb, NP, kl);     // X V g        (n x nl)
    {
      const bool own = sa.per_point != 0;
      double2* gv = sa.grad_v + (own ? (long long)p * nl * n : k * (sa.v_ks ? (long long)nl * n : 0));
      for (long long e = tid; e < M2; e += kThreads) {
        const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
        if (r < nl && c < n) grad_put(gv + (long long)r * n + c, cadd(Aq[e], cconj(Bp[(long long)c * NP + r])), own);
      }
      __syncthreads();  // Aq and Bp are rewritten next
    }
    // P = g H01, Q = H10 g
    gemm_to<false, false>(Pk, Gb, H01b, NP, kl);
    if (h10) gemm_to<false, false>(Aq, H10b, Gb, NP, kl);
    else gemm_to<true, false>(Aq, H01b, Gb, NP, kl);
    copy_mat(Bp, Pk, NP);
    copy_mat(Lam, Gbar, NP);
    // Smith doubling for Lam - Q Lam P = gbar
    int status = kOk, it = 0;
    for (;;) {
      ++it;
      gemm_to<false, false>(Tt, Aq, Lam, NP, kl);
      gemm_add<false, false>(Lam, Tt, Bp, NP, kl);
      gemm_to<false, false>(Aq2, Aq, Aq, NP, kl);
      gemm_to<false, false>(Bp2, Bp, Bp, NP, kl);
      double2* t = Aq;
      Aq = Aq2;
      Aq2 = t;
      t = Bp;
      Bp = Bp2;
      Bp2 = t;
      double m = 0.0;
      int bad = 0;
      for (long long e = tid; e < M2; e += kThreads) {
        const double2 a = Aq[e], b = Bp[e], l = Lam[e];
        bad |= !(cfinite(a) && cfinite(b) && cfinite(l));
        m = fmax(m, fmax(fmax(fabs(a.x), fabs(a.y)), fmax(fabs(b.x), fabs(b.y))));
      }
      if (block_any(bad)) {
        status = kNonFinite;
        break;
      }
      m = block_max(m, red);
      if (m < sa.tol) break;
      if (it >= sa.maxiter) {
        status = kMaxIter;
        break;
      }
    }
    if (status == kOk) {
      gemm_to<false, false>(Tt, Lam, Gb, NP, kl);    // Lam g
      gemm_to<false, false>(T1, Gb, Tt, NP, kl);     // H00bar = g Lam g
      if (h10) gemm_to<false, false>(Tt, Gb, H10b, NP, kl);   // g H10
      else gemm_to<false, true>(Tt, Gb, H01b, NP, kl);
      gemm_to<false, false>(T2, Tt, T1, NP, kl);     // H01bar = g H10 H00bar
      gemm_to<false, false>(Aq2, H01b, Gb, NP, kl);  // H01 g
      gemm_to<false, false>(Tt, T1, Aq2, NP, kl);    // H10bar = H00bar H01 g
      const bool own = sa.per_point != 0;
      const long long slot = own ? (long long)p : k;
      double2* g00 = sa.grad_h00 + slot * nl * nl;
      double2* g01 = sa.grad_h01 + slot * nl * nl;
      double2* g10 = sa.grad_h10 ? sa.grad_h10 + slot * nl * nl : nullptr;
      for (long long e = tid; e < M2; e += kThreads) {
        const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
        if (r < nl && c < nl) {
          grad_put(g00 + r * nl + c, T1[e], own);
          if (h10) {
            grad_put(g01 + r * nl + c, T2[e], own);
            if (g10) grad_put(g10 + r * nl + c, Tt[e], own);
          } else {
            grad_put(g01 + r * nl + c, cadd(T2[e], cconj(Tt[(long long)c * NP + r])), own);
          }
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      if (sa.status_out) sa.status_out[p] = status;
      if (sa.iters_out) sa.iters_out[p] = it;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ full device G --
// Every block of G = A^-1 for one point (negfpy core/negf.py:253-303 builds it
// densely with SuperLU).  One left sweep keeps g^L_i, W_i = g^L_i C_i and
// V_i = C_i^H g^L_i; the diagonal follows backwards without further inverses,
//   G_{L-1,L-1} = g^L_{L-1},  G_ii = g^L_i + W_i G_{i+1,i+1} V_i,
// and the off-diagonal blocks by walking each column up and each row left,
//   G_ij = W_i G_{i+1,j},  G_ji = G_{j,i+1} V_i   (i < j).
// Blocks are written into G_out[p] (row-major, order L n); Sigma_L and Sigma_R
// (n x n) into their outputs.
__device__ void put_block(double2* Gp, long long dim, int bi, int bj, const double2* src, int n, int NP) {
  for (int e = threadIdx.x; e < n * n; e += kThreads) {
    const int r = e / n, c = e - r * n;
    Gp[((long long)bi * n + r) * dim + (long long)bj * n + c] = src[(long long)r * NP + c];
  }
}

__global__ void __launch_bounds__(kThreads, 2) rgf_full_f64_kernel(FullArgs fa, int NP, double2* ws) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const GJS sh = carve(smraw, NP);
  __shared__ int s_point;
  const RgfArgs& a = fa.r;
  const int n = a.n, L = a.L, tid = threadIdx.x;
  const int kch = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  const long long dim = (long long)L * n;
  double2* base = ws + (long long)blockIdx.x * ((6 + 3LL * L) * M2 + 2LL * n * n);
  double2 *Cb = base, *B1 = base + M2, *B2 = base + 2 * M2, *Xs = base + 3 * M2, *P0 = base + 4 * M2,
          *P1 = base + 5 * M2;
  double2* gl = base + 6 * M2;              // L slots: g^L_i, then G_ii
  double2* Ws = gl + (long long)L * M2;     // L slots: W_i
  double2* Vs = Ws + (long long)L * M2;     // L slots: V_i
  double2* sigL = Vs + (long long)L * M2;
  double2* sigR = sigL + (long long)n * n;

  for (;;) {
    if (tid == 0) s_point = (int)atomicAdd(a.counter, 1u);
    __syncthreads();
    const int p = s_point;
    __syncthreads();
    if (p >= a.batch) break;
    const int lst = a.lead_status ? a.lead_status[p] : 0;
    if (lst != kOk) {
      if (tid == 0 && a.status_out) a.status_out[p] = lst;
      continue;
    }
    const long long k = a.kidx ? (long long)a.kidx[p] : 0;
    RgfPoint q;
    q.n = n;
    q.nl = a.nl;
    q.nr = a.nr;
    q.L = L;
    q.D = a.D + k * a.d_ks;
    q.d_ls = a.d_ls;
    q.C = a.C + k * a.c_ks;
    q.c_ls = a.c_ls;
    q.VL = a.VL + k * a.vl_ks;
    q.VR = a.VR + k * a.vr_ks;
    q.gL = a.gL + (long long)p * a.gl_ps;
    q.gR = a.gR + (long long)p * a.gr_ps;
    q.z = z_of(a.omega[p], a.eta_dev[p]);
    self_energies(q, NP, B1, B2, Xs, sigL, sigR);
    for (int e = tid; e < n * n; e += kThreads) {
      fa.sigL_out[(long long)p * n * n + e] = sigL[e];
      fa.sigR_out[(long long)p * n * n + e] = sigR[e];
    }
    auto Dl = [&](int l) { return q.D + (long long)l * q.d_ls; };
    int status = kOk;
    // left sweep with W_l, V_l
    form_m<false, false>(gl, nullptr, nullptr, Dl(0), sigL, L == 1 ? sigR : nullptr, q.z, n, NP, kch);
    status = invert_into(gl, Xs, n, NP, sh);
    for (int l = 1; l < L && status == kOk; ++l) {
      load_pad(Cb, q.C + (long long)(l - 1) * q.c_ls, n, n, NP, 0.0);
      __syncthreads();
      gemm_to<false, false>(Ws + (l - 1) * M2, gl + (l - 1) * M2, Cb, NP, kch);
      gemm_to<true, false>(Vs + (l - 1) * M2, Cb, gl + (l - 1) * M2, NP, kch);
      form_m<true, false>(gl + l * M2, Cb, Ws + (l - 1) * M2, Dl(l), l == L - 1 ? sigR : nullptr, nullptr, q.z, n,
                          NP, kch);
      status = invert_into(gl + l * M2, Xs, n, NP, sh);
    }
    if (status == kOk) {
      double2* Gp = fa.G + (long long)p * dim * dim;
      // diagonal, backwards: G_ii = g^L_i + W_i G_{i+1,i+1} V_i (into the g^L slot)
      put_block(Gp, dim, L - 1, L - 1, gl + (L - 1) * M2, n, NP);
      for (int i = L - 2; i >= 0; --i) {
        gemm_to<false, false>(P0, Ws + i * M2, gl + (i + 1) * M2, NP, kch);
        gemm_to<false, false>(P1, P0, Vs + i * M2, NP, kch);
        double2* gi = gl + i * M2;
        for (long long e = tid; e < M2; e += kThreads) gi[e] = cadd(gi[e], P1[e]);
        __syncthreads();
        put_block(Gp, dim, i, i, gi, n, NP);
      }
      // columns up and rows left from each diagonal block
      for (int j = 1; j < L; ++j) {
        const double2* src = gl + j * M2;
        double2 *x = P0, *y = P1;
        for (int i = j - 1; i >= 0; --i) {
          gemm_to<false, false>(x, Ws + i * M2, src, NP, kch);   // G_ij = W_i G_{i+1,j}
          put_block(Gp, dim, i, j, x, n, NP);
          src = x;
          x = (x == P0) ? B1 : P0;
        }
        src = gl + j * M2;
        for (int i = j - 1; i >= 0; --i) {
          gemm_to<false, false>(y, src, Vs + i * M2, NP, kch);   // G_ji = G_{j,i+1} V_i
          put_block(Gp, dim, j, i, y, n, NP);
          src = y;
          y = (y == P1) ? B2 : P1;
        }
        __syncthreads();
      }
    }
    __syncthreads();
    if (tid == 0 && a.status_out) a.status_out[p] = status;
    __syncthreads();
  }
}

// ---------------------------------------------------------------- launchers --
size_t smem_bytes(int np) { return ((gjs_bytes(np) + 15) / 16) * 16 + 40 * 8; }

template <typename K>
static int occupancy_grid(K kernel, int np) {
  const size_t sm = smem_bytes(np);
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) return -3;
  int nb = 0, dev = 0, nsm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, kThreads, sm) != cudaSuccess || nb <= 0) return -3;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nb * nsm;
}

}  // namespace glob

int sr_global_grid(int np) { return glob::occupancy_grid(glob::sr_f64_global_kernel, np); }
int rgf_global_grid(int np) { return glob::occupancy_grid(glob::rgf_f64_global_kernel, np); }
size_t sr_global_ws_bytes(int np, int grid) { return (size_t)grid * 7 * np * np * 16; }
size_t rgf_global_ws_bytes(int np, int n, int grid) { return (size_t)grid * (6 * (size_t)np * np + 2 * (size_t)n * n) * 16; }

int sr_f64_global_launch(const SrArgs& a, int np, int grid, double2* ws, unsigned* counter, cudaStream_t st) {
  if (a.batch <= 0) return 0;
  glob::sr_f64_global_kernel<<<grid, glob::kThreads, glob::smem_bytes(np), st>>>(a, np, ws, counter);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

size_t grad_ws_bytes(int np, int n, int L, int grid) {
  return (size_t)grid * ((14 + 2 * (size_t)L) * np * np + 2 * (size_t)n * n) * 16;
}
int grad_grid(int np) {
  const int g = glob::occupancy_grid(glob::rgf_grad_f64_kernel, np);
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return g > 2 * nsm ? 2 * nsm : g;  // two blocks per SM bound the 2L-slot workspace
}
size_t full_ws_bytes(int np, int n, int L, int grid) {
  return (size_t)grid * ((6 + 3 * (size_t)L) * np * np + 2 * (size_t)n * n) * 16;
}
int full_grid(int np) {
  const int g = glob::occupancy_grid(glob::rgf_full_f64_kernel, np);
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return g > 2 * nsm ? 2 * nsm : g;
}
int full_f64_launch(const FullArgs& fa, int np, int grid, double2* ws, cudaStream_t st) {
  if (fa.r.batch <= 0) return 0;
  glob::rgf_full_f64_kernel<<<grid, glob::kThreads, glob::smem_bytes(np), st>>>(fa, np, ws);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
size_t sgf_adj_ws_bytes(int np, int grid) { return (size_t)grid * 15 * (size_t)np * np * 16; }
int sgf_adj_grid(int np) {
  const int g = glob::occupancy_grid(glob::sgf_adjoint_f64_kernel, np);
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return g > 2 * nsm ? 2 * nsm : g;
}
int sgf_adj_launch(const SgfAdjArgs& sa, int np, int grid, double2* ws, cudaStream_t st) {
  if (sa.batch <= 0) return 0;
  glob::sgf_adjoint_f64_kernel<<<grid, glob::kThreads, glob::smem_bytes(np), st>>>(sa, np, ws);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}
int grad_f64_launch(const GradArgs& ga, int np, int grid, double2* ws, cudaStream_t st) {
  if (ga.r.batch <= 0) return 0;
  glob::rgf_grad_f64_kernel<<<grid, glob::kThreads, glob::smem_bytes(np), st>>>(ga, np, ws);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

int rgf_f64_global_launch(const RgfArgs& a, int np, int grid, double2* ws, cudaStream_t st) {
  if (a.batch <= 0) return 0;
  glob::rgf_f64_global_kernel<<<grid, glob::kThreads, glob::smem_bytes(np), st>>>(a, np, ws);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace negf

namespace negf {
int global_order(int n) {
  if (n <= 48 || n > 256) return 0;
  return (n + 15) / 16 * 16;
}
}  // namespace negf
