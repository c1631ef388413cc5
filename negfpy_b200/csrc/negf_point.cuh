// Per-point bodies of the global-workspace FP64 kernels, shared by the
// single-system kernels (negf_f64_global.cu) and the uneven batch kernel
// (negf_batch.cu).  Each function is executed by a whole thread block on one
// (omega, k) point, in workspace buffers the caller owns; every call ends
// with the block synchronised.
#pragma once
#include "negf_common.cuh"
#include "negf_tiles.cuh"

namespace negf {
namespace glob {

// Sancho-Rubio decimation of one point (negfpy core/surface_gf.py:18-81):
// the recurrence, the stopping rule max(|alpha|, |beta|) < tol and the final
// g = (z - eps_s)^-1 of sr_f64_kernel.  `buf` holds 7 NP x NP buffers.
// Returns the status; *iters the sweeps taken; *g the buffer holding the
// padded surface GF (row stride NP), valid when the status is kOk.
static __device__ int sr_point(int n, int NP, const double2* h00, const double2* h01, const double2* h10,
                               double2 z, double tol, int maxiter, double2* buf, const GJS& sh, double* red,
                               int* iters, double2** g) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const int np16 = NP >> 4, ntiles = np16 * np16, kch = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  double2 *pa = buf, *pb = buf + M2, *pe = buf + 2 * M2, *pes = buf + 3 * M2;
  double2 *f0 = buf + 4 * M2, *f1 = buf + 5 * M2, *f2 = buf + 6 * M2;
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
  const double tol2 = tol * tol;
  double2* pg = nullptr;
  for (it = 1; it <= maxiter; ++it) {
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
    if (block_any(bad)) {
      status = sr_failure_status(it, n, h00, h01, h10, z);
      break;
    }
    const double emax = block_max(e2, red);
    if (emax < tol2) {
      converged = true;
      break;
    }
  }
  if (status == kOk && !converged) {
    status = kMaxIter;
    it = maxiter;
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
  *iters = it;
  *g = pg;
  return status;
}

// One point of the device solve, with the blocks of its k already selected.
struct RgfPoint {
  int n, nl, nr, L;
  const double2* D;  long long d_ls;   // onsite block l at D + l*d_ls (n x n)
  const double2* C;  long long c_ls;   // coupling block l at C + l*c_ls
  const double2* VL;                   // n x nl
  const double2* VR;                   // n x nr
  const double2* gL;                   // nl x nl surface GF, row stride nl
  const double2* gR;                   // nr x nr
  double2 z;
};

// Sigma = V g V^H for both contacts into sigL / sigR (n x n each), FP64.
// B0, B1, B2: NP x NP scratch.
static __device__ void self_energies(const RgfPoint& q, int NP, double2* B0, double2* B1, double2* B2,
                                     double2* sigL, double2* sigR) {
  const int warp = threadIdx.x >> 5, np16 = NP >> 4, ntiles = np16 * np16, n = q.n;
  for (int side = 0; side < 2; ++side) {
    const int nl = side ? q.nr : q.nl;
    const int lch = (nl + 7) >> 3;
    const double2* V = side ? q.VR : q.VL;
    const double2* g = side ? q.gR : q.gL;
    double2* S = side ? sigR : sigL;
    load_pad(B0, V, n, nl, NP, 0.0);
    load_pad(B1, g, nl, nl, NP, 0.0);
    __syncthreads();
    for (int tt = warp; tt < ntiles; tt += kWarps) {
      const Tile T = tile_of(tt, np16);
      Acc c;
      tile_mm<false, false>(c, B0, NP, B1, NP, lch, T);
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) B2[(long long)tr(T, qq) * NP + tc(T, j, qq)] = c.get(j, qq);
    }
    __syncthreads();
    for (int tt = warp; tt < ntiles; tt += kWarps) {
      const Tile T = tile_of(tt, np16);
      Acc c;
      tile_mm<false, true>(c, B2, NP, B0, NP, lch, T);
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) {
          const int r = tr(T, qq), cc = tc(T, j, qq);
          if (r < n && cc < n) S[r * n + cc] = c.get(j, qq);
        }
    }
    __syncthreads();
  }
}

// T = Re sum_ij (Gamma_L G Gamma_R)_ij conj(G_ij) in FP64 for G = G_{0,L-1}
// in G64 (NP x NP); GL, GR, U: NP x NP scratch.  Returns the block-wide sum.
static __device__ double trace_t(int n, int NP, const double2* sigL, const double2* sigR, const double2* G64,
                                 double2* GL, double2* GR, double2* U, double* red) {
  const int tid = threadIdx.x, warp = tid >> 5, np16 = NP >> 4, ntiles = np16 * np16, kch = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  for (long long e = tid; e < M2; e += kThreads) {
    const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
    double2 gl = make_double2(0.0, 0.0), gr = gl;
    if (r < n && c < n) {
      double2 d = csub(sigL[r * n + c], cconj(sigL[c * n + r]));
      gl = make_double2(-d.y, d.x);
      d = csub(sigR[r * n + c], cconj(sigR[c * n + r]));
      gr = make_double2(-d.y, d.x);
    }
    GL[e] = gl;
    GR[e] = gr;
  }
  __syncthreads();
  for (int tt = warp; tt < ntiles; tt += kWarps) {
    const Tile T = tile_of(tt, np16);
    Acc c1;
    tile_mm<false, false>(c1, GL, NP, G64, NP, kch, T);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) U[(long long)tr(T, q) * NP + tc(T, j, q)] = c1.get(j, q);
  }
  __syncthreads();
  double t = 0.0;
  for (int tt = warp; tt < ntiles; tt += kWarps) {
    const Tile T = tile_of(tt, np16);
    Acc c1;
    tile_mm<false, false>(c1, U, NP, GR, NP, kch, T);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double2 g = G64[(long long)tr(T, q) * NP + tc(T, j, q)];
        t += c1.re[j][q] * g.x + c1.im[j][q] * g.y;
      }
  }
  return block_sum(t, red);
}

// Sigma, left-connected RGF sweep and trace of one point in FP64 (negfpy
// core/negf.py:72-357).  `buf`: 6 NP x NP buffers followed by 2 n x n.
// Returns the status; *t the transmission when kOk.
static __device__ int rgf_point_f64(const RgfPoint& q, int NP, double2* buf, const GJS& sh, double* red, double* t) {
  const int n = q.n, L = q.L, tid = threadIdx.x, warp = tid >> 5;
  const int np16 = NP >> 4, ntiles = np16 * np16, kch = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  double2* sigL = buf + 6 * M2;
  double2* sigR = sigL + (long long)n * n;
  double2 *pg = buf, *pc = buf + M2, *bW = buf + 2 * M2, *bU = buf + 3 * M2, *bG0 = buf + 4 * M2,
          *bX = buf + 5 * M2;
  const double2 z = q.z;
  self_energies(q, NP, bW, bX, bU, sigL, sigR);
  // Layer 0: g_0 = (z - D_0 - Sigma_L [- Sigma_R when L == 1])^-1 = G_{0,0}.
  for (long long e = tid; e < M2; e += kThreads) {
    const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
    double2 v;
    if (r < n && c < n) {
      v = csub(cneg(q.D[r * n + c]), sigL[r * n + c]);
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
      load_pad(pc, q.C + (long long)(l - 1) * q.c_ls, n, n, NP, 0.0);
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
          for (int qq = 0; qq < 4; ++qq) {
            const long long e = (long long)tr(T, qq) * NP + tc(T, j, qq);
            bW[e] = c1.get(j, qq);
            bU[e] = c2.get(j, qq);
          }
      }
      __syncthreads();
      // M = z - D_l - C^H W [- Sigma_R on the last layer] into the old g buffer
      const double2* Dl = q.D + (long long)l * q.d_ls;
      const bool last = (l == L - 1);
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc c1;
        tile_mm<true, false>(c1, pc, NP, bW, NP, kch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int qq = 0; qq < 4; ++qq) {
            const int r = tr(T, qq), cc = tc(T, j, qq);
            double2 v;
            if (r < n && cc < n) {
              v = csub(cneg(Dl[r * n + cc]), c1.get(j, qq));
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
          for (int qq = 0; qq < 4; ++qq) bG0[(long long)tr(T, qq) * NP + tc(T, j, qq)] = c1.get(j, qq);
      }
      __syncthreads();
    }
  }
  double tval = 0.0;
  if (status == kOk) {
    tval = trace_t(n, NP, sigL, sigR, bG0, pc, bW, bU, red);
    if (!isfinite(tval)) status = kNonFinite;
  } else {
    __syncthreads();
  }
  *t = tval;
  return status;
}

}  // namespace glob
}  // namespace negf
