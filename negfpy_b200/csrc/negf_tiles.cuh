// Warp-tile building blocks of the global-workspace kernels: FP64 DMMA
// complex products on 16 x 16 tiles whose fragments are loaded from
// row-major global (L2-resident) matrices, padded loads, and the blocked
// Gauss-Jordan inverse between two global buffers.  Shared by the
// FP64 kernels and by the FP64 parts (self-energies, trace) of the
// mixed-precision device solve.
#pragma once
#include "negf_common.cuh"

namespace negf {
namespace glob {

constexpr int kWarps = 8;
constexpr int kThreads = 32 * kWarps;

__device__ __forceinline__ double2 z_of(double w, double e) {
  return make_double2(__dsub_rn(__dmul_rn(w, w), __dmul_rn(e, e)), __dmul_rn(2.0 * w, e));
}

__device__ __forceinline__ void dmma(double (&d)[4], const double (&a)[4], double b0, double b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b0), "d"(b1));
}
__device__ __forceinline__ void cmma(double (&cr)[4], double (&ci)[4], const double (&ar)[4], const double (&ai)[4],
                                     const double (&br)[2], const double (&bi)[2]) {
  dmma(cr, ar, br[0], br[1]);
  dmma(cr, ai, -bi[0], -bi[1]);
  dmma(ci, ar, bi[0], bi[1]);
  dmma(ci, ai, br[0], br[1]);
}

struct Acc {
  double re[2][4], im[2][4];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) re[j][q] = im[j][q] = 0.0;
  }
  __device__ __forceinline__ double2 get(int j, int q) const { return make_double2(re[j][q], im[j][q]); }
};

// Tile geometry: tile t of the (NP/16)^2 grid, lane (g, t4).
struct Tile {
  int m0, n0, g, t;
};
__device__ __forceinline__ Tile tile_of(int tt, int np16) {
  Tile T;
  const int l = threadIdx.x & 31;
  T.g = l >> 2;
  T.t = l & 3;
  T.m0 = (tt / np16) * 16;
  T.n0 = (tt % np16) * 16;
  return T;
}
__device__ __forceinline__ int tr(const Tile& T, int q) { return T.m0 + T.g + 8 * (q >> 1); }
__device__ __forceinline__ int tc(const Tile& T, int j, int q) { return T.n0 + 8 * j + 2 * T.t + (q & 1); }

// acc = op(A) op(B) for one 16 x 16 tile, contraction over kch chunks of 8
// (ADD: acc += op(A) op(B)).  AC / BC: operand is the conjugate transpose of
// the stored matrix.  lda / ldb: row strides of the stored matrices.
template <bool AC, bool BC, bool ADD = false>
__device__ __forceinline__ void tile_mm(Acc& c, const double2* __restrict__ A, int lda, const double2* __restrict__ B,
                                        int ldb, int kch, const Tile& T) {
  if (!ADD) c.zero();
  for (int kc = 0; kc < kch; ++kc) {
    const int k0 = kc * 8;
    double ar[4], ai[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = T.m0 + T.g + 8 * (q & 1), k = k0 + T.t + 4 * (q >> 1);
      const double2 v = AC ? A[(long long)k * lda + r] : A[(long long)r * lda + k];
      ar[q] = v.x;
      ai[q] = AC ? -v.y : v.y;
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      double br[2], bi[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int k = k0 + T.t + 4 * q, cc = T.n0 + 8 * j + T.g;
        const double2 v = BC ? B[(long long)cc * ldb + k] : B[(long long)k * ldb + cc];
        br[q] = v.x;
        bi[q] = BC ? -v.y : v.y;
      }
      cmma(c.re[j], c.im[j], ar, ai, br, bi);
    }
  }
}

// Global nr x nc matrix -> padded NP x NP buffer (zeros outside, `diag` on the
// padding diagonal).
__device__ __forceinline__ void load_pad(double2* dst, const double2* __restrict__ src, int nr, int nc, int NP,
                                         double diag) {
  for (long long e = threadIdx.x; e < (long long)NP * NP; e += kThreads) {
    const int r = (int)(e / NP), c = (int)(e - (long long)r * NP);
    double2 v = (r < nr && c < nc) ? src[(long long)r * nc + c] : make_double2(0.0, 0.0);
    if (r == c && (r >= nr || c >= nc)) v = make_double2(diag, 0.0);
    dst[e] = v;
  }
}

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
  unsigned* key;  // [8][kWarps] each warp's pivot key of each panel column
};
__host__ __device__ inline size_t gjs_bytes(int np) {
  return (size_t)2 * np * 8 * 16 + 3 * np * 4 + 8 * kWarps * 4;
}
// Pivot key of a panel column: the maximum of the kWarps warp keys in `row`
// (16-byte aligned).  Each warp posts its key in its own slot, so no shared
// atomics are needed.
__device__ __forceinline__ unsigned key_max(const unsigned* row) {
  static_assert(kWarps % 4 == 0, "key slots are read 4 at a time");
  unsigned k = 0u;
#pragma unroll
  for (int w = 0; w < kWarps; w += 4) {
    const uint4 v = *reinterpret_cast<const uint4*>(row + w);
    k = max(k, max(max(v.x, v.y), max(v.z, v.w)));
  }
  return k;
}
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
static __device__ int gj_invert_global(double2* X, double2* Y, int n, int NP, const GJS& sh, double2** out) {
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
    key0 = __reduce_max_sync(0xffffffffu, key0);
    if (lane == 0) sh.key[warp] = key0;
    __syncthreads();
    double2 lam = make_double2(1.0, 0.0);
    // Bit i: row (tid >> 3) + 32 i (this thread's rows; its column is
    // tid & 7) was a pivot row of this panel.
    static_assert(kThreads == 256, "rows of a thread are 32 apart");
    unsigned used_rows = 0u;
    for (int j = 0; j < jmax; ++j) {
      const unsigned key = key_max(sh.key + j * kWarps);
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
      if ((pr & 31) == (tid >> 3)) used_rows |= 1u << (pr >> 5);
      unsigned nk = 0u;
      for (int e = tid, i = 0; e < PE; e += kThreads, ++i) {
        const int r = e >> 3, c = e & 7;
        const bool isp = (r == pr);
        const double2 fv = P[r * 8 + j], mv = P[pr * 8 + c], av = P[e];
        const double2 bb = isp ? cneg(lam) : fv;
        const double2 b = make_double2(bb.x * sc, bb.y * sc);
        const double2 m = (c == j) ? lam : mv;
        double2 v = cneg(cmul(b, m));
        if (!isp && c != j) cfma(v, ps, av);
        Pn[e] = v;
        if (c == j + 1 && r >= k0 && r < n && !((used_rows >> i) & 1u)) nk = max(nk, pivot_key8(v, r));
      }
      lam = cmul(lam, ps);
      if (j + 1 < jmax) {
        nk = __reduce_max_sync(0xffffffffu, nk);
        if (lane == 0) sh.key[(j + 1) * kWarps + warp] = nk;
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

}  // namespace glob
}  // namespace negf
