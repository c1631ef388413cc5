// FP64 kernels for block orders 49..256 (padded to NP, a multiple of 16).
//
// One point's matrices do not fit one SM's shared memory beyond n = 48, so
// here they live in a per-block workspace in global memory (L2-resident for
// n <= 96 with one block per SM, HBM beyond) and the blocks are persistent:
// each takes points from an atomic counter and several blocks share an SM,
// so one point's latency-bound pivot steps overlap another's products.
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
#include "negf_tiles.cuh"

namespace negf {
namespace glob {

// ---------------------------------------------------------- Gauss-Jordan --
__device__ __forceinline__ unsigned pivot_key8(double2 v, int r) {
  const unsigned ha = (unsigned)__double2hiint(v.x) & 0x7fffffffu;
  const unsigned hb = (unsigned)__double2hiint(v.y) & 0x7fffffffu;
  const unsigned hm = ha > hb ? ha : hb;
  return (hm & ~255u) | (unsigned)(255 - r);
}
__device__ __forceinline__ double2 crecip_smith(double2 v) {
  if (fabs(v.x) >= fabs(v.y)) {
    const double r = v.y / v.x;
    const double i = 1.0 / fma(v.y, r, v.x);
    return make_double2(i, -r * i);
  }
  const double r = v.x / v.y;
  const double i = 1.0 / fma(v.x, r, v.y);
  return make_double2(r * i, -i);
}

// Shared scratch of the inversion for order NP: panel ping-pong (2 x NP x 8),
// permutation bookkeeping and the panel keys.
struct GJS {
  double2* panel;
  int* sig;
  int* siginv;
  int* pivlog;
  unsigned* key;
};
__host__ __device__ inline size_t gjs_bytes(int np) { return (size_t)2 * np * 8 * 16 + 3 * np * 4 + 8 * 4; }
__device__ __forceinline__ GJS carve(unsigned char* base, int np) {
  GJS s;
  s.panel = reinterpret_cast<double2*>(base);
  s.sig = reinterpret_cast<int*>(base + (size_t)2 * np * 8 * 16);
  s.siginv = s.sig + np;
  s.pivlog = s.siginv + np;
  s.key = reinterpret_cast<unsigned*>(s.pivlog + np);
  return s;
}

// Inverse of the leading n x n block of X (padding = identity), NP <= 256,
// using Y as the second global buffer; *out is the buffer with the inverse.
// Same algorithm as gj_invert of the shared-memory kernels (see there): the
// n x 8 panels are factored in shared memory by the whole block with a
// division-free lambda-scaled rule and look-ahead pivot keys (top bits of
// max(|re|, |im|), row index in the low 8 bits: the column maximum up to a
// relative 2^-12), the rank-8 update writes the next global buffer in the new
// row order, and the interchanges are undone by a final column gather.
__device__ int gj_invert_global(double2* X, double2* Y, int n, int NP, const GJS& sh, double2** out) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int np16 = NP >> 4, ntiles = np16 * np16;
  const int PE = NP * 8;
  double2* cur = X;
  double2* nxt = Y;
  for (int k0 = 0; k0 < n; k0 += 8) {
    const int jmax = (n - k0) < 8 ? (n - k0) : 8;
    double2* P = sh.panel;
    double2* Pn = sh.panel + PE;
    unsigned key0 = 0u;
    for (int e = tid; e < PE; e += kThreads) {
      const int r = e >> 3, c = e & 7;
      const double2 v = cur[(long long)r * NP + k0 + c];
      P[e] = v;
      if (c == 0 && r >= k0 && r < n) key0 = max(key0, pivot_key8(v, r));
    }
    for (int r = tid; r < NP; r += kThreads) {
      sh.sig[r] = r;
      sh.siginv[r] = r;
    }
    if (tid < 8) sh.key[tid] = 0u;
    __syncthreads();
    key0 = __reduce_max_sync(0xffffffffu, key0);
    if (lane == 0 && key0) atomicMax(&sh.key[0], key0);
    __syncthreads();
    double2 lam = make_double2(1.0, 0.0);
    for (int j = 0; j < jmax; ++j) {
      const unsigned key = sh.key[j];
      if ((key >> 20) >= 0x7ffu) return kNonFinite;
      if ((key >> 8) == 0u) return kSingular;
      const int pr = 255 - (int)(key & 255u);
      const int ex = (int)(key >> 20);
      const double sc = (ex != 0 && ex < 2046) ? __hiloint2double((2046 - ex) << 20, 0) : 1.0;
      if (tid == 0) {
        const int k = k0 + j;
        const int bl = sh.siginv[pr];
        const int pa = sh.sig[k];
        sh.sig[k] = pr;
        sh.sig[bl] = pa;
        sh.siginv[pr] = k;
        sh.siginv[pa] = bl;
        sh.pivlog[k] = bl;
      }
      const double2 piv = P[pr * 8 + j];
      const double2 ps = make_double2(piv.x * sc, piv.y * sc);
      unsigned nk = 0u;
      for (int e = tid; e < PE; e += kThreads) {
        const int r = e >> 3, c = e & 7;
        const bool isp = (r == pr);
        // rows already used as pivots in this panel are sig[k0..k0+j]
        const double2 fv = P[r * 8 + j], mv = P[pr * 8 + c], av = P[e];
        const double2 bb = isp ? cneg(lam) : fv;
        const double2 b = make_double2(bb.x * sc, bb.y * sc);
        const double2 m = (c == j) ? lam : mv;
        double2 v = cneg(cmul(b, m));
        if (!isp && c != j) cfma(v, ps, av);
        Pn[e] = v;
        if (c == j + 1 && r >= k0 && r < n) {
          bool used = isp;
          for (int i = 0; i < j; ++i) used = used || (sh.sig[k0 + i] == r);
          if (!used) nk = max(nk, pivot_key8(v, r));
        }
      }
      lam = cmul(lam, ps);
      if (j + 1 < jmax) {
        nk = __reduce_max_sync(0xffffffffu, nk);
        if (lane == 0 && nk) atomicMax(&sh.key[j + 1], nk);
      }
      __syncthreads();
      double2* t = P;
      P = Pn;
      Pn = t;
    }
    // rank-8 update of the whole matrix
    const double2 il = crecip_smith(lam);
    for (int tt = warp; tt < ntiles; tt += kWarps) {
      const Tile T = tile_of(tt, np16);
      Acc c;
      int srow[2];
      bool inpanel[2];
#pragma unroll
      for (int ri = 0; ri < 2; ++ri) {
        const int r = T.m0 + T.g + 8 * ri;
        srow[ri] = sh.sig[r];
        inpanel[ri] = r >= k0 && r < k0 + jmax;
      }
#pragma unroll
      for (int j2 = 0; j2 < 2; ++j2)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double2 v = cur[(long long)srow[q >> 1] * NP + tc(T, j2, q)];
          c.re[j2][q] = inpanel[q >> 1] ? 0.0 : v.x;
          c.im[j2][q] = inpanel[q >> 1] ? 0.0 : v.y;
        }
      double ar[4], ai[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int kk = T.t + 4 * (q >> 1);
        const double2 v = cmul(P[srow[q & 1] * 8 + kk], il);
        ar[q] = v.x;
        ai[q] = v.y;
      }
      const int kk0 = T.t, kk1 = T.t + 4;
      const int pr0 = kk0 < jmax ? sh.sig[k0 + kk0] : 0, pr1 = kk1 < jmax ? sh.sig[k0 + kk1] : 0;
#pragma unroll
      for (int j2 = 0; j2 < 2; ++j2) {
        const int cc = T.n0 + 8 * j2 + T.g;
        const double2 v0 = cur[(long long)pr0 * NP + cc], v1 = cur[(long long)pr1 * NP + cc];
        double br[2], bi[2];
        br[0] = kk0 < jmax ? v0.x : 0.0;
        bi[0] = kk0 < jmax ? v0.y : 0.0;
        br[1] = kk1 < jmax ? v1.x : 0.0;
        bi[1] = kk1 < jmax ? v1.y : 0.0;
        cmma(c.re[j2], c.im[j2], ar, ai, br, bi);
      }
#pragma unroll
      for (int j2 = 0; j2 < 2; ++j2)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = tr(T, q), cc = tc(T, j2, q);
          double2 v = c.get(j2, q);
          if (cc >= k0 && cc < k0 + 8) v = cmul(P[srow[q >> 1] * 8 + (cc - k0)], il);
          nxt[(long long)r * NP + cc] = v;
        }
    }
    __syncthreads();
    double2* t = cur;
    cur = nxt;
    nxt = t;
  }
  // Column map: column c of the inverse = column t_{n-1}(...t_0(c)) of cur.
  // pivlog holds the partners; build the map for every column at once.
  __syncthreads();
  for (int c = tid; c < NP; c += kThreads) {
    int s = c;
    for (int k = 0; k < n; ++k) {
      const int b = sh.pivlog[k];
      s = (s == k) ? b : ((s == b) ? k : s);
    }
    sh.sig[c] = s;
  }
  __syncthreads();
  for (long long e = tid; e < (long long)NP * NP; e += kThreads) {
    const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
    nxt[e] = cur[(long long)r * NP + sh.sig[c]];
  }
  __syncthreads();
  *out = nxt;
  return kOk;
}

// ------------------------------------------------------------ Sancho-Rubio --
// Workspace per block: 7 NP x NP buffers (alpha, beta, eps, eps_s, three free).
__global__ void __launch_bounds__(kThreads) sr_f64_global_kernel(SrArgs a, int NP, double2* ws, unsigned* counter) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const GJS sh = carve(smraw, NP);
  double* red = reinterpret_cast<double*>(smraw + ((gjs_bytes(NP) + 15) / 16) * 16);
  __shared__ int s_point;
  const int n = a.n, tid = threadIdx.x, warp = tid >> 5;
  const int np16 = NP >> 4, ntiles = np16 * np16, kch = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  double2* base = ws + (long long)blockIdx.x * 7 * M2;

  for (;;) {
    if (tid == 0) s_point = (int)atomicAdd(counter, 1u);
    __syncthreads();
    const int p = s_point;
    __syncthreads();
    if (p >= a.batch) break;
    double2 *pa = base, *pb = base + M2, *pe = base + 2 * M2, *pes = base + 3 * M2;
    double2 *f0 = base + 4 * M2, *f1 = base + 5 * M2, *f2 = base + 6 * M2;
    const long long kset = a.kidx ? (long long)a.kidx[p] : 0;
    const double2* h00 = a.h00 + kset * a.lead_stride;
    const double2* h01 = a.h01 + kset * a.lead_stride;
    const double2* h10 = a.h10 ? a.h10 + kset * a.lead_stride : nullptr;
    const double w = a.omega[p];
    const double2 z = z_of(w, a.eta[p]);
    for (long long e = tid; e < M2; e += kThreads) {
      const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
      const bool in = r < n && c < n;
      const double2 e0 = in ? h00[r * n + c] : make_double2(0.0, 0.0);
      pe[e] = e0;
      pes[e] = e0;
      pa[e] = in ? h01[r * n + c] : make_double2(0.0, 0.0);
      pb[e] = in ? (h10 ? h10[r * n + c] : cconj(h01[c * n + r])) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    int status = kOk, it = 0;
    bool converged = false;
    const double tol2 = a.tol * a.tol;
    double2* pg = nullptr;
    for (it = 1; it <= a.maxiter; ++it) {
      for (long long e = tid; e < M2; e += kThreads) {
        const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
        double2 v;
        if (r < n && c < n) v = (r == c) ? csub(z, pe[e]) : cneg(pe[e]);
        else v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        f0[e] = v;
      }
      __syncthreads();
      status = gj_invert_global(f0, f1, n, NP, sh, &pg);
      if (status != kOk) break;
      double2* pag = (pg == f0) ? f1 : f0;
      double2* pbg = f2;
      // alpha g, beta g
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc c;
        tile_mm<false, false>(c, pa, NP, pg, NP, kch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) pag[(long long)tr(T, q) * NP + tc(T, j, q)] = c.get(j, q);
        tile_mm<false, false>(c, pb, NP, pg, NP, kch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) pbg[(long long)tr(T, q) * NP + tc(T, j, q)] = c.get(j, q);
      }
      __syncthreads();
      // eps_s += (alpha g) beta ; eps += (alpha g) beta + (beta g) alpha ;
      // beta' = (beta g) beta into the free g buffer
      int bad = 0;
      double e2 = 0.0;
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc c1, c2;
        tile_mm<false, false>(c1, pag, NP, pb, NP, kch, T);
        tile_mm<false, false>(c2, pbg, NP, pa, NP, kch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const long long e = (long long)tr(T, q) * NP + tc(T, j, q);
            const double2 x1 = c1.get(j, q);
            const double2 es = cadd(pes[e], x1), ee = cadd(cadd(pe[e], x1), c2.get(j, q));
            pes[e] = es;
            pe[e] = ee;
            bad |= !cfinite(es) || !cfinite(ee);
          }
        tile_mm<false, false>(c1, pbg, NP, pb, NP, kch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const double2 v = c1.get(j, q);
            bad |= !cfinite(v);
            e2 = fmax(e2, cabs2(v));
            pg[(long long)tr(T, q) * NP + tc(T, j, q)] = v;
          }
      }
      __syncthreads();
      // alpha' = (alpha g) alpha into the beta g buffer (free now)
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc c1;
        tile_mm<false, false>(c1, pag, NP, pa, NP, kch, T);
        __syncwarp();
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const double2 v = c1.get(j, q);
            bad |= !cfinite(v);
            e2 = fmax(e2, cabs2(v));
            pbg[(long long)tr(T, q) * NP + tc(T, j, q)] = v;
          }
      }
      __syncthreads();
      {
        double2* oa = pa;
        double2* ob = pb;
        pa = pbg;  // alpha'
        pb = pg;   // beta'
        f0 = oa;
        f1 = ob;
        f2 = pag;
      }
      if (block_any(bad)) { status = kNonFinite; break; }
      const double emax = block_max(e2, red);
      if (emax < tol2) { converged = true; break; }
    }
    if (status == kOk && !converged) {
      status = kMaxIter;
      it = a.maxiter;
    }
    if (status == kOk) {
      for (long long e = tid; e < M2; e += kThreads) {
        const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
        double2 v;
        if (r < n && c < n) v = (r == c) ? csub(z, pes[e]) : cneg(pes[e]);
        else v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        f0[e] = v;
      }
      __syncthreads();
      status = gj_invert_global(f0, f1, n, NP, sh, &pg);
    }
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
__global__ void __launch_bounds__(kThreads) rgf_f64_global_kernel(RgfArgs a, int NP, double2* ws) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const GJS sh = carve(smraw, NP);
  double* red = reinterpret_cast<double*>(smraw + ((gjs_bytes(NP) + 15) / 16) * 16);
  __shared__ int s_point;
  const int n = a.n, L = a.L, tid = threadIdx.x, warp = tid >> 5;
  const int np16 = NP >> 4, ntiles = np16 * np16, kch = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  double2* base = ws + (long long)blockIdx.x * (6 * M2 + 2LL * n * n);
  double2* sigL = base + 6 * M2;
  double2* sigR = sigL + (long long)n * n;

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
    // g_l, padded coupling, W = g C, U = G0 C, G0, second inversion buffer
    double2 *pg = base, *pc = base + M2, *bW = base + 2 * M2, *bU = base + 3 * M2, *bG0 = base + 4 * M2,
            *bX = base + 5 * M2;
    const long long k = a.kidx ? (long long)a.kidx[p] : 0;
    const double2 z = z_of(a.omega[p], a.eta_dev[p]);
    const double2* D = a.D + k * a.d_ks;
    const double2* C = a.C + k * a.c_ks;

    // Sigma = V g V^H for both contacts (V padded to NP x NP in bW, g in bX).
    for (int side = 0; side < 2; ++side) {
      const int nl = side ? a.nr : a.nl;
      const int lch = (nl + 7) >> 3;
      const double2* V = side ? a.VR + k * a.vr_ks : a.VL + k * a.vl_ks;
      const double2* g = side ? a.gR + (long long)p * a.gr_ps : a.gL + (long long)p * a.gl_ps;
      double2* S = side ? sigR : sigL;
      load_pad(bW, V, n, nl, NP, 0.0);
      load_pad(bX, g, nl, nl, NP, 0.0);
      __syncthreads();
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc c;
        tile_mm<false, false>(c, bW, NP, bX, NP, lch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) bU[(long long)tr(T, q) * NP + tc(T, j, q)] = c.get(j, q);
      }
      __syncthreads();
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc c;
        tile_mm<false, true>(c, bU, NP, bW, NP, lch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int r = tr(T, q), cc = tc(T, j, q);
            if (r < n && cc < n) S[r * n + cc] = c.get(j, q);
          }
      }
      __syncthreads();
    }
    // Layer 0: g_0 = (z - D_0 - Sigma_L [- Sigma_R when L == 1])^-1 = G_{0,0}.
    for (long long e = tid; e < M2; e += kThreads) {
      const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
      double2 v;
      if (r < n && c < n) {
        v = csub(cneg(D[r * n + c]), sigL[r * n + c]);
        if (L == 1) v = csub(v, sigR[r * n + c]);
        if (r == c) v = cadd(v, z);
      } else {
        v = make_double2(r == c ? 1.0 : 0.0, 0.0);
      }
      pg[e] = v;
    }
    __syncthreads();
    double2* inv = nullptr;
    int status = gj_invert_global(pg, bX, n, NP, sh, &inv);
    if (status == kOk) {
      if (inv != pg) {
        bX = pg;
        pg = inv;
      }
      for (long long e = tid; e < M2; e += kThreads) bG0[e] = pg[e];
      for (int l = 1; l < L && status == kOk; ++l) {
        load_pad(pc, C + (long long)(l - 1) * a.c_ls, n, n, NP, 0.0);
        __syncthreads();
        // W = g_{l-1} C, U = G_{0,l-1} C
        for (int tt = warp; tt < ntiles; tt += kWarps) {
          const Tile T = tile_of(tt, np16);
          Acc c1, c2;
          tile_mm<false, false>(c1, pg, NP, pc, NP, kch, T);
          tile_mm<false, false>(c2, bG0, NP, pc, NP, kch, T);
#pragma unroll
          for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const long long e = (long long)tr(T, q) * NP + tc(T, j, q);
              bW[e] = c1.get(j, q);
              bU[e] = c2.get(j, q);
            }
        }
        __syncthreads();
        // M = z - D_l - C^H W [- Sigma_R on the last layer] into the old g buffer
        const double2* Dl = D + (long long)l * a.d_ls;
        const bool last = (l == L - 1);
        for (int tt = warp; tt < ntiles; tt += kWarps) {
          const Tile T = tile_of(tt, np16);
          Acc c1;
          tile_mm<true, false>(c1, pc, NP, bW, NP, kch, T);
#pragma unroll
          for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int r = tr(T, q), cc = tc(T, j, q);
              double2 v;
              if (r < n && cc < n) {
                v = csub(cneg(Dl[r * n + cc]), c1.get(j, q));
                if (last) v = csub(v, sigR[r * n + cc]);
                if (r == cc) v = cadd(v, z);
              } else {
                v = make_double2(r == cc ? 1.0 : 0.0, 0.0);
              }
              pg[(long long)r * NP + cc] = v;
            }
        }
        __syncthreads();
        status = gj_invert_global(pg, bX, n, NP, sh, &inv);
        if (status != kOk) break;
        if (inv != pg) {
          bX = pg;
          pg = inv;
        }
        // G_{0,l} = U g_l
        for (int tt = warp; tt < ntiles; tt += kWarps) {
          const Tile T = tile_of(tt, np16);
          Acc c1;
          tile_mm<false, false>(c1, bU, NP, pg, NP, kch, T);
#pragma unroll
          for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) bG0[(long long)tr(T, q) * NP + tc(T, j, q)] = c1.get(j, q);
        }
        __syncthreads();
      }
    }
    double tval = 0.0;
    if (status == kOk) {
      for (long long e = tid; e < M2; e += kThreads) {
        const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
        double2 gl = make_double2(0.0, 0.0), gr = gl;
        if (r < n && c < n) {
          double2 d = csub(sigL[r * n + c], cconj(sigL[c * n + r]));
          gl = make_double2(-d.y, d.x);
          d = csub(sigR[r * n + c], cconj(sigR[c * n + r]));
          gr = make_double2(-d.y, d.x);
        }
        pc[e] = gl;
        bW[e] = gr;
      }
      __syncthreads();
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc c1;
        tile_mm<false, false>(c1, pc, NP, bG0, NP, kch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) bU[(long long)tr(T, q) * NP + tc(T, j, q)] = c1.get(j, q);
      }
      __syncthreads();
      double t = 0.0;
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc c1;
        tile_mm<false, false>(c1, bU, NP, bW, NP, kch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const double2 g = bG0[(long long)tr(T, q) * NP + tc(T, j, q)];
            t += c1.re[j][q] * g.x + c1.im[j][q] * g.y;
          }
      }
      tval = block_sum(t, red);
      if (!isfinite(tval)) status = kNonFinite;
    } else {
      __syncthreads();
    }
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
__global__ void __launch_bounds__(kThreads) rgf_grad_f64_kernel(GradArgs ga, int NP, double2* ws) {
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
    double2* gdk = ga.grad_d + k * (long long)L * n * n;
    double2* gck = ga.grad_c + k * (long long)(L > 1 ? L - 1 : 1) * n * n;
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
    // 4. first block row and the adjoint blocks
    for (int i = 0; i < L && status == kOk; ++i) {
      gemm_to<false, false>(Ac, gl + i * M2, Y, NP, kch);
      gemm_to<false, false>(Xa, Ac, G0c, NP, kch);
      for (long long e = tid; e < M2; e += kThreads) {
        const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
        if (r < n && c < n) {
          const double2 v = Xa[e];
          atomic_cadd(gdk + (long long)i * n * n + r * n + c, make_double2(wgt * v.x, wgt * v.y));
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
            atomic_cadd(gck + (long long)(i - 1) * n * n + r * n + c, make_double2(wgt * v.x, wgt * v.y));
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
  return g > nsm ? nsm : g;  // one block per SM bounds the 2L-slot workspace
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
