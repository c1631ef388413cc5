// Warp-tile building blocks of the global-workspace kernels: FP64 DMMA
// complex products on 16 x 16 tiles whose fragments are loaded from
// row-major global (L2-resident) matrices, and padded loads.  Shared by the
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

// acc = op(A) op(B) for one 16 x 16 tile, contraction over kch chunks of 8.
// AC / BC: operand is the conjugate transpose of the stored matrix.
// lda / ldb: row strides of the stored matrices.
template <bool AC, bool BC>
__device__ __forceinline__ void tile_mm(Acc& c, const double2* __restrict__ A, int lda, const double2* __restrict__ B,
                                        int ldb, int kch, const Tile& T) {
  c.zero();
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

}  // namespace glob
}  // namespace negf
