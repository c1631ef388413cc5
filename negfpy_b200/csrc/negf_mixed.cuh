// Mixed-precision device solve, per point: FP32 sweep on 3 x TF32
// tensor-core products and an FP32 Gauss-Jordan; FP64 self-energies,
// broadenings and trace.  Shared by rgf_mixed_kernel (negf_mixed.cu) and the
// uneven batch kernel (negf_batch.cu).
#pragma once
#include "negf_common.cuh"
#include "negf_point.cuh"
#include "negf_tcprod.cuh"
#include "negf_tiles.cuh"

namespace negf {
namespace mixed {

using glob::kThreads;
using glob::kWarps;
using glob::Tile;
using glob::tc;
using glob::tile_of;
using glob::tr;

__device__ __forceinline__ float2 fneg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 fmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 to_f(double2 v) { return make_float2((float)v.x, (float)v.y); }

// ------------------------------------------------------ 3 x TF32 products --
__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// A fragment (16 x 8) of a complex matrix, split: re/im x hi/lo.
struct AFrag {
  unsigned rh[4], rl[4], ih[4], il[4];
};
// B fragment (8 x 8): re, im and -im, each hi/lo.
struct BFrag {
  unsigned rh[2], rl[2], ih[2], il[2], nih[2], nil[2];
};
__device__ __forceinline__ void set_a(AFrag& f, int q, float2 v) {
  split_tf32(v.x, f.rh[q], f.rl[q]);
  split_tf32(v.y, f.ih[q], f.il[q]);
}
__device__ __forceinline__ void set_b(BFrag& f, int q, float2 v) {
  split_tf32(v.x, f.rh[q], f.rl[q]);
  split_tf32(v.y, f.ih[q], f.il[q]);
  f.nih[q] = f.ih[q] ^ 0x80000000u;
  f.nil[q] = f.il[q] ^ 0x80000000u;
}
// c += a b for one m16n8 complex tile: real = ar br - ai bi, imag = ar bi + ai br,
// each real product as lo*hi + hi*lo + hi*hi (small terms first).
__device__ __forceinline__ void cmma3(float (&cr)[4], float (&ci)[4], const AFrag& a, const BFrag& b) {
  mma_tf32(cr, a.rl, b.rh[0], b.rh[1]);
  mma_tf32(cr, a.rh, b.rl[0], b.rl[1]);
  mma_tf32(cr, a.il, b.nih[0], b.nih[1]);
  mma_tf32(cr, a.ih, b.nil[0], b.nil[1]);
  mma_tf32(cr, a.rh, b.rh[0], b.rh[1]);
  mma_tf32(cr, a.ih, b.nih[0], b.nih[1]);
  mma_tf32(ci, a.rl, b.ih[0], b.ih[1]);
  mma_tf32(ci, a.rh, b.il[0], b.il[1]);
  mma_tf32(ci, a.il, b.rh[0], b.rh[1]);
  mma_tf32(ci, a.ih, b.rl[0], b.rl[1]);
  mma_tf32(ci, a.rh, b.ih[0], b.ih[1]);
  mma_tf32(ci, a.ih, b.rh[0], b.rh[1]);
}

struct Acc32 {
  float re[2][4], im[2][4];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) re[j][q] = im[j][q] = 0.f;
  }
  __device__ __forceinline__ float2 get(int j, int q) const { return make_float2(re[j][q], im[j][q]); }
};

// acc = op(A) op(B) for one 16 x 16 tile (FP32 matrices, row stride ld),
// contraction over kch chunks of 8 (ADD: acc += op(A) op(B)); AC / BC:
// conjugate-transposed operand.
template <bool AC, bool BC, bool ADD = false>
__device__ __forceinline__ void tile_mm32(Acc32& c, const float2* __restrict__ A, const float2* __restrict__ B, int ld,
                                          int kch, const Tile& T) {
  if (!ADD) c.zero();
  for (int kc = 0; kc < kch; ++kc) {
    const int k0 = kc * 8;
    AFrag a;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = T.m0 + T.g + 8 * (q & 1), k = k0 + T.t + 4 * (q >> 1);
      float2 v = AC ? A[(long long)k * ld + r] : A[(long long)r * ld + k];
      if (AC) v.y = -v.y;
      set_a(a, q, v);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      BFrag b;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int k = k0 + T.t + 4 * q, cc = T.n0 + 8 * j + T.g;
        float2 v = BC ? B[(long long)cc * ld + k] : B[(long long)k * ld + cc];
        if (BC) v.y = -v.y;
        set_b(b, q, v);
      }
      // The chunk's three passes start from zero and are added with a
      // round-to-nearest FP32 add: the tensor cores' own accumulation
      // truncates, and accumulating every chunk inside them biases |c| low.
      float pr[4] = {0.f, 0.f, 0.f, 0.f}, pi[4] = {0.f, 0.f, 0.f, 0.f};
      cmma3(pr, pi, a, b);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        c.re[j][q] = __fadd_rn(c.re[j][q], pr[q]);
        c.im[j][q] = __fadd_rn(c.im[j][q], pi[q]);
      }
    }
  }
}

// ------------------------------------------------------- FP32 Gauss-Jordan --
// Same algorithm as glob::gj_invert_global: 8-column panels in shared memory,
// division-free lambda-scaled elimination, look-ahead integer pivot keys (top
// bits of max(|re|, |im|) as FP32 bit patterns, row index in the low 8 bits),
// rank-8 update between two global buffers, final column gather.
struct GJS32 {
  float2* panel;
  int* sig;
  int* siginv;
  int* pivlog;
  unsigned* key;  // [8][kWarps] each warp's pivot key of each panel column
};
__host__ __device__ inline size_t gjs32_bytes(int np) {
  return (size_t)2 * np * 8 * 8 + 3 * np * 4 + 8 * glob::kWarps * 4;
}
__device__ __forceinline__ GJS32 carve32(unsigned char* base, int np) {
  GJS32 s;
  s.panel = reinterpret_cast<float2*>(base);
  s.sig = reinterpret_cast<int*>(base + (size_t)2 * np * 8 * 8);
  s.siginv = s.sig + np;
  s.pivlog = s.siginv + np;
  s.key = reinterpret_cast<unsigned*>(s.pivlog + np);
  return s;
}
__device__ __forceinline__ unsigned pivot_key32(float2 v, int r) {
  const unsigned ha = __float_as_uint(v.x) & 0x7fffffffu;
  const unsigned hb = __float_as_uint(v.y) & 0x7fffffffu;
  const unsigned hm = ha > hb ? ha : hb;
  return (hm & ~255u) | (unsigned)(255 - r);
}
// 1 / v by Smith's algorithm (R. L. Smith, CACM 5(8), 1962).
__device__ __forceinline__ float2 crecip_smith32(float2 v) {
  if (fabsf(v.x) >= fabsf(v.y)) {
    const float r = v.y / v.x;
    const float i = 1.0f / fmaf(v.y, r, v.x);
    return make_float2(i, -r * i);
  }
  const float r = v.x / v.y;
  const float i = 1.0f / fmaf(v.x, r, v.y);
  return make_float2(r * i, -i);
}

static __device__ int gj_invert32(float2* X, float2* Y, int n, int NP, const GJS32& sh, float2** out) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int np16 = NP >> 4, ntiles = np16 * np16;
  const int PE = NP * 8;
  float2* cur = X;
  float2* nxt = Y;
  for (int k0 = 0; k0 < n; k0 += 8) {
    const int jmax = (n - k0) < 8 ? (n - k0) : 8;
    float2* P = sh.panel;
    float2* Pn = sh.panel + PE;
    unsigned key0 = 0u;
    for (int e = tid; e < PE; e += kThreads) {
      const int r = e >> 3, c = e & 7;
      const float2 v = cur[(long long)r * NP + k0 + c];
      P[e] = v;
      if (c == 0 && r >= k0 && r < n) key0 = max(key0, pivot_key32(v, r));
    }
    for (int r = tid; r < NP; r += kThreads) {
      sh.sig[r] = r;
      sh.siginv[r] = r;
    }
    key0 = __reduce_max_sync(0xffffffffu, key0);
    if (lane == 0) sh.key[warp] = key0;
    __syncthreads();
    float2 lam = make_float2(1.f, 0.f);
    // Bit i: row (tid >> 3) + 32 i (this thread's rows; its column is
    // tid & 7) was a pivot row of this panel.
    static_assert(kThreads == 256, "rows of a thread are 32 apart");
    unsigned used_rows = 0u;
    for (int j = 0; j < jmax; ++j) {
      const unsigned key = glob::key_max(sh.key + j * glob::kWarps);
      if ((key >> 23) >= 0xffu) return kNonFinite;
      if ((key >> 8) == 0u) return kSingular;
      const int pr = 255 - (int)(key & 255u);
      const int ex = (int)(key >> 23);
      const float sc = (ex != 0 && ex < 254) ? __uint_as_float((unsigned)(254 - ex) << 23) : 1.0f;
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
      const float2 piv = P[pr * 8 + j];
      const float2 ps = make_float2(piv.x * sc, piv.y * sc);
      if ((pr & 31) == (tid >> 3)) used_rows |= 1u << (pr >> 5);
      unsigned nk = 0u;
      for (int e = tid, i = 0; e < PE; e += kThreads, ++i) {
        const int r = e >> 3, c = e & 7;
        const bool isp = (r == pr);
        const float2 fv = P[r * 8 + j], mv = P[pr * 8 + c], av = P[e];
        const float2 bb = isp ? fneg(lam) : fv;
        const float2 b = make_float2(bb.x * sc, bb.y * sc);
        const float2 m = (c == j) ? lam : mv;
        float2 v = fneg(fmulc(b, m));
        if (!isp && c != j) cfma(v, ps, av);
        Pn[e] = v;
        if (c == j + 1 && r >= k0 && r < n && !((used_rows >> i) & 1u)) nk = max(nk, pivot_key32(v, r));
      }
      lam = fmulc(lam, ps);
      if (j + 1 < jmax) {
        nk = __reduce_max_sync(0xffffffffu, nk);
        if (lane == 0) sh.key[(j + 1) * glob::kWarps + warp] = nk;
      }
      __syncthreads();
      float2* t = P;
      P = Pn;
      Pn = t;
    }
    // rank-8 update of the whole matrix
    const float2 il = crecip_smith32(lam);
    for (int tt = warp; tt < ntiles; tt += kWarps) {
      const Tile T = tile_of(tt, np16);
      Acc32 c;
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
          const float2 v = cur[(long long)srow[q >> 1] * NP + tc(T, j2, q)];
          c.re[j2][q] = inpanel[q >> 1] ? 0.f : v.x;
          c.im[j2][q] = inpanel[q >> 1] ? 0.f : v.y;
        }
      AFrag a;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int kk = T.t + 4 * (q >> 1);
        set_a(a, q, fmulc(P[srow[q & 1] * 8 + kk], il));
      }
      const int kk0 = T.t, kk1 = T.t + 4;
      const int pr0 = kk0 < jmax ? sh.sig[k0 + kk0] : 0, pr1 = kk1 < jmax ? sh.sig[k0 + kk1] : 0;
#pragma unroll
      for (int j2 = 0; j2 < 2; ++j2) {
        const int cc = T.n0 + 8 * j2 + T.g;
        const float2 v0 = cur[(long long)pr0 * NP + cc], v1 = cur[(long long)pr1 * NP + cc];
        BFrag b;
        set_b(b, 0, kk0 < jmax ? v0 : make_float2(0.f, 0.f));
        set_b(b, 1, kk1 < jmax ? v1 : make_float2(0.f, 0.f));
        float pr[4] = {0.f, 0.f, 0.f, 0.f}, pi[4] = {0.f, 0.f, 0.f, 0.f};
        cmma3(pr, pi, a, b);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          c.re[j2][q] = __fadd_rn(c.re[j2][q], pr[q]);
          c.im[j2][q] = __fadd_rn(c.im[j2][q], pi[q]);
        }
      }
#pragma unroll
      for (int j2 = 0; j2 < 2; ++j2)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = tr(T, q), cc = tc(T, j2, q);
          float2 v = c.get(j2, q);
          if (cc >= k0 && cc < k0 + 8) v = fmulc(P[srow[q >> 1] * 8 + (cc - k0)], il);
          nxt[(long long)r * NP + cc] = v;
        }
    }
    __syncthreads();
    float2* t = cur;
    cur = nxt;
    nxt = t;
  }
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

// FP64 n x n (row stride n) -> FP32 padded NP x NP, zeros outside.
__device__ __forceinline__ void load_pad32(float2* dst, const double2* __restrict__ src, int n, int NP) {
  for (long long e = threadIdx.x; e < (long long)NP * NP; e += kThreads) {
    const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
    dst[e] = (r < n && c < n) ? to_f(src[(long long)r * n + c]) : make_float2(0.f, 0.f);
  }
}

// Workspace per block: 4 NP x NP FP64 buffers (V / g / V g for the
// self-energies, then Gamma_L, Gamma_R, G widened, Gamma_L G), Sigma_L and
// Sigma_R (n x n FP64), and 6 NP x NP FP32 buffers (g_l, C, W, U, G_0, the
// second inversion buffer).
__host__ __device__ inline size_t mixed_ws_elems64(int np, int n) { return 4 * (size_t)np * np + 2 * (size_t)n * n; }
__host__ __device__ inline size_t mixed_ws_bytes_per_block(int np, int n) {
  return mixed_ws_elems64(np, n) * 16 + 6 * (size_t)np * np * 8;
}

// Sigma, Gamma and trace in FP64, the RGF sweep in FP32, for one point whose
// blocks are selected in q.  `blk` is the block's workspace
// (mixed_ws_bytes_per_block(NP, n) bytes).  Returns the status; *t the
// transmission when kOk.  TC: the sweep's four products per layer run on
// tcgen05 (tc::cprod with the block's context *tcx; NP <= 128), otherwise on
// mma.sync; the inversions run on mma.sync either way.
template <bool TC = false>
static __device__ int rgf_point_mixed(const glob::RgfPoint& q, int NP, unsigned char* blk, const GJS32& sh,
                                      double* red, double* t, tc::Ctx* tcx = nullptr) {
  const int n = q.n, L = q.L, tid = threadIdx.x, warp = tid >> 5;
  const int np16 = NP >> 4, ntiles = np16 * np16, kch = (n + 7) >> 3;
  const long long M2 = (long long)NP * NP;
  double2* d64 = reinterpret_cast<double2*>(blk);
  double2 *B0 = d64, *B1 = d64 + M2, *B2 = d64 + 2 * M2, *B3 = d64 + 3 * M2;
  double2* sigL = d64 + 4 * M2;
  double2* sigR = sigL + (long long)n * n;
  float2* f32 = reinterpret_cast<float2*>(blk + mixed_ws_elems64(NP, n) * 16);
  const double2 z = q.z;
  const double2* D = q.D;
  const double2* C = q.C;
  float2 *pg = f32, *pc = f32 + M2, *bW = f32 + 2 * M2, *bU = f32 + 3 * M2, *bG0 = f32 + 4 * M2,
         *bX = f32 + 5 * M2;
  glob::self_energies(q, NP, B0, B1, B2, sigL, sigR);
  // FP32 sweep.  Layer 0: g_0 = (z - D_0 - Sigma_L [- Sigma_R when L == 1])^-1.
  for (long long e = tid; e < M2; e += kThreads) {
    const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
    float2 v;
    if (r < n && c < n) {
      double2 w = csub(cneg(D[r * n + c]), sigL[r * n + c]);
      if (L == 1) w = csub(w, sigR[r * n + c]);
      if (r == c) w = cadd(w, z);
      v = to_f(w);
    } else {
      v = make_float2(r == c ? 1.f : 0.f, 0.f);
    }
    pg[e] = v;
  }
  __syncthreads();
  float2* inv = nullptr;
  int status = gj_invert32(pg, bX, n, NP, sh, &inv);
  if (status == kOk) {
    if (inv != pg) {
      bX = pg;
      pg = inv;
    }
    for (long long e = tid; e < M2; e += kThreads) bG0[e] = pg[e];
    for (int l = 1; l < L && status == kOk; ++l) {
      load_pad32(pc, C + (long long)(l - 1) * q.c_ls, n, NP);
      __syncthreads();
      const double2* Dl = D + (long long)l * q.d_ls;
      const bool last = (l == L - 1);
      if constexpr (TC) {
        // W = g C, U = G_0 C, X = C^H W on tcgen05; M formed from X below
        bool ok = tc::cprod<false, false>(bW, pg, pc, NP, *tcx);
        ok = tc::cprod<false, false>(bU, bG0, pc, NP, *tcx) && ok;
        ok = tc::cprod<true, false>(bX, pc, bW, NP, *tcx) && ok;
        if (!ok) {
          status = kNonFinite;
          break;
        }
        for (long long e = tid; e < M2; e += kThreads) {
          const int r = (int)(e / NP), cc = (int)(e - (long long)r * NP);
          float2 v;
          if (r < n && cc < n) {
            double2 w = cneg(Dl[r * n + cc]);
            if (last) w = csub(w, sigR[r * n + cc]);
            if (r == cc) w = cadd(w, z);
            const float2 x = bX[e];
            v = make_float2((float)(w.x - (double)x.x), (float)(w.y - (double)x.y));
          } else {
            v = make_float2(r == cc ? 1.f : 0.f, 0.f);
          }
          pg[e] = v;
        }
        __syncthreads();
      } else {
      // W = g_{l-1} C, U = G_{0,l-1} C
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc32 c1, c2;
        tile_mm32<false, false>(c1, pg, pc, NP, kch, T);
        tile_mm32<false, false>(c2, bG0, pc, NP, kch, T);
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
      // M = z - D_l - C^H W [- Sigma_R on the last layer] into the old g buffer;
      // the FP64 terms are combined in FP64 before the rounding.
      for (int tt = warp; tt < ntiles; tt += kWarps) {
        const Tile T = tile_of(tt, np16);
        Acc32 c1;
        tile_mm32<true, false>(c1, pc, bW, NP, kch, T);
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int qq = 0; qq < 4; ++qq) {
            const int r = tr(T, qq), cc = tc(T, j, qq);
            float2 v;
            if (r < n && cc < n) {
              double2 w = cneg(Dl[r * n + cc]);
              if (last) w = csub(w, sigR[r * n + cc]);
              if (r == cc) w = cadd(w, z);
              v = make_float2((float)(w.x - (double)c1.re[j][qq]), (float)(w.y - (double)c1.im[j][qq]));
            } else {
              v = make_float2(r == cc ? 1.f : 0.f, 0.f);
            }
            pg[(long long)r * NP + cc] = v;
          }
      }
      __syncthreads();
      }
      status = gj_invert32(pg, bX, n, NP, sh, &inv);
      if (status != kOk) break;
      if (inv != pg) {
        bX = pg;
        pg = inv;
      }
      // G_{0,l} = U g_l
      if constexpr (TC) {
        if (!tc::cprod<false, false>(bG0, bU, pg, NP, *tcx)) {
          status = kNonFinite;
          break;
        }
      } else {
        for (int tt = warp; tt < ntiles; tt += kWarps) {
          const Tile T = tile_of(tt, np16);
          Acc32 c1;
          tile_mm32<false, false>(c1, bU, pg, NP, kch, T);
#pragma unroll
          for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) bG0[(long long)tr(T, qq) * NP + tc(T, j, qq)] = c1.get(j, qq);
        }
        __syncthreads();
      }
    }
  }
  // FP64: Gamma_L, Gamma_R, G widened, T = Re sum (Gamma_L G Gamma_R)_ij conj(G_ij).
  double tval = 0.0;
  if (status == kOk) {
    for (long long e = tid; e < M2; e += kThreads) {
      const float2 gv = bG0[e];
      B2[e] = make_double2((double)gv.x, (double)gv.y);
    }
    __syncthreads();
    tval = glob::trace_t(n, NP, sigL, sigR, B2, B0, B1, B3, red);
    if (!isfinite(tval)) status = kNonFinite;
  } else {
    __syncthreads();
  }
  *t = tval;
  return status;
}

}  // namespace mixed
}  // namespace negf
