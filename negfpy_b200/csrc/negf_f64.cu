// FP64 kernels of the per-(omega, k) phonon NEGF path.
//
// One thread block owns one (omega, k) point at a time.  Blocks of order
// n <= 48 live entirely in shared memory, zero-padded to NP in {16, 32, 48}.
// Complex products run on the FP64 tensor path: mma.sync m16n8k8 f64, four
// real MMAs per complex tile (re += ar br - ai bi, im += ar bi + ai br).
// Warp w owns the 16 x 16 output region (16*(w / T), 16*(w % T)), T = NP/16,
// as two 16 x 8 MMA tiles; in every elementwise phase (Gauss-Jordan updates,
// epilogues, register-resident matrices) a thread owns exactly the eight
// elements its MMA accumulators hold, so no data moves between phases.
//
// Shared matrices are stored as interleaved (re, im) pairs, row-major with
// row stride NP, and the column index XOR-swizzled per row (see sidx) so the
// A-fragment pattern (2 rows x 4 columns per 8 lanes) and the B-fragment /
// conjugate-transpose pattern (4 rows x 2 columns) are both conflict-free.
//
//   sr_f64_kernel   Sancho-Rubio decimation (negfpy core/surface_gf.py:18-81):
//                   alpha, beta, g = (z - eps)^-1, alpha g, beta g in shared
//                   memory; eps and eps_s in registers.  Epilogues: g_s,
//                   surface DOS (core/dos.py:31-61).
//   rgf_f64_kernel  Sigma = V g V^H for both contacts (core/negf.py:72-97),
//                   left-connected recursive Green's function sweep for
//                   G_{0,L-1} of A = z - D - Sigma (core/negf.py:141-250,
//                   replacing the SuperLU solve at :353), Gamma = i(S - S^H)
//                   (:115-116) and T = Re Tr[Gamma_L G Gamma_R G^H] (:356).
//   *_scalar_kernel the same for 1 x 1 blocks (the monatomic chain), one
//                   thread per point.
#include <cstdio>

#include "negf_common.cuh"
#include "negf_f64.h"

namespace negf {

// z = (omega + i eta)^2 with the two products rounded separately, as the
// reference's complex power does (no fused multiply-add in the real part).
__device__ __forceinline__ double2 z_of(double w, double e) {
  return make_double2(__dsub_rn(__dmul_rn(w, w), __dmul_rn(e, e)), __dmul_rn(2.0 * w, e));
}

template <int NP>
struct Geo {
  static constexpr int T = NP / 16;     // 16-row tiles per side
  static constexpr int NW = T * T;      // tile warps, one 16 x 16 region each
  // Warps per block: a multiple of the SM's 4 sub-partitions.  At NP = 48
  // the 3 warps beyond the 9 tile warps own no tile; they take part in the
  // Gauss-Jordan panel (one element per thread) and its bookkeeping.
  static constexpr int NWB = (NW % 4 == 0 || NW == 1) ? NW : (NW + 3) / 4 * 4;
  static constexpr int NTH = 32 * NWB;  // threads
  static constexpr int MAT = NP * NP;   // complex elements per matrix buffer
};

// Row-dependent XOR swizzle of the column index (bits 0-2), values
// {0, 5, 2, 7, 1, 4, 3, 6} for r mod 8 = 0..7.  With 16-byte elements and
// phases of 8 lanes it makes every access pattern used here conflict-free:
// A fragments (rows r, r+1 x 4 columns: bit 2 differs), B fragments and
// conjugate-transpose walks (4 rows x 2 columns: bits 2-1 distinct),
// accumulator stores (rows r, r+1 x even columns: bit 0 differs) and column
// walks (8 rows: all distinct).
__device__ __forceinline__ int swz(int r) { return (int)((0xCE1EA8u >> (3 * (r & 7))) & 7u); }
template <int NP>
__device__ __forceinline__ int sidx(int r, int c) { return r * NP + (c ^ swz(r)); }

// Lane geometry of the warp's 16 x 16 region.
struct Lane {
  int g, t, m0, n0;
};
// Warps without a tile get tile 0's geometry, so that any fragment address
// they form stays in range; tile-owned work masks them out (Split::jt).
template <int NP>
__device__ __forceinline__ Lane lane_geo() {
  const int w0 = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int w = w0 < Geo<NP>::NW ? w0 : 0;
  Lane L;
  L.g = l >> 2;
  L.t = l & 3;
  L.m0 = (w / Geo<NP>::T) * 16;
  L.n0 = (w % Geo<NP>::T) * 16;
  return L;
}
// Element (row, col) held in accumulator slot q of tile j (8 slots per thread).
__device__ __forceinline__ int own_r(const Lane& L, int q) { return L.m0 + L.g + 8 * (q >> 1); }
__device__ __forceinline__ int own_c(const Lane& L, int j, int q) { return L.n0 + 8 * j + 2 * L.t + (q & 1); }

// Complex accumulators of the warp's two 16 x 8 tiles.
struct CAcc {
  double re[2][4], im[2][4];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) re[j][q] = im[j][q] = 0.0;
  }
  __device__ __forceinline__ double2 get(int j, int q) const { return make_double2(re[j][q], im[j][q]); }
};

__device__ __forceinline__ void dmma(double (&d)[4], const double (&a)[4], double b0, double b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b0), "d"(b1));
}

// Fragment addressing.  Chunk k0 (a multiple of 8) never changes an index
// modulo 8, so every fragment address is a loop-invariant base plus k0
// (row-major walk) or k0 * NP (column walk).
//   A = S     : (m0+g+8(q&1), k0+t+4(q>>1)) -> base + k0
//   A = S^H   : S(k0+t+4(q>>1), m0+g+8(q&1)) -> base + k0*NP
//   B = S     : S(k0+t+4q, nb+g)             -> base + k0*NP
//   B = S^H   : S(nb+g, k0+t+4q)             -> base + k0
template <int NP, bool CT>
__device__ __forceinline__ void a_bases(const Lane& L, int (&base)[4]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int r = L.m0 + L.g + 8 * (q & 1), kk = L.t + 4 * (q >> 1);
    base[q] = CT ? sidx<NP>(kk, r) : sidx<NP>(r, kk);
  }
}
template <int NP, bool CT>
__device__ __forceinline__ void b_bases(const Lane& L, int (&base)[2][2]) {
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int kk = L.t + 4 * q, c = L.n0 + 8 * j + L.g;
      base[j][q] = CT ? sidx<NP>(c, kk) : sidx<NP>(kk, c);
    }
}
template <int NP, bool CT>
__device__ __forceinline__ void load_a(const double2* __restrict__ S, const int (&base)[4], int k0, double (&ar)[4],
                                       double (&ai)[4]) {
  const int off = CT ? k0 * NP : k0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double2 v = S[base[q] + off];
    ar[q] = v.x;
    ai[q] = CT ? -v.y : v.y;
  }
}
template <int NP, bool CT>
__device__ __forceinline__ void load_b(const double2* __restrict__ S, const int (&base)[2], int k0, double (&br)[2],
                                       double (&bi)[2]) {
  const int off = CT ? k0 : k0 * NP;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const double2 v = S[base[q] + off];
    br[q] = v.x;
    bi[q] = CT ? -v.y : v.y;
  }
}
__device__ __forceinline__ void cmma(double (&cr)[4], double (&ci)[4], const double (&ar)[4], const double (&ai)[4],
                                     const double (&br)[2], const double (&bi)[2]) {
  dmma(cr, ar, br[0], br[1]);
  dmma(cr, ai, -bi[0], -bi[1]);
  dmma(ci, ar, bi[0], bi[1]);
  dmma(ci, ai, br[0], br[1]);
}

// c = op(A) op(B) over the first kch chunks of 8 (the rest is zero padding).
// jm: warp-uniform mask of the two 16 x 8 halves (j) to compute.
template <int NP, bool AC, bool BC>
__device__ __forceinline__ void cmm(CAcc& c, const double2* A, const double2* B, int kch, const Lane& L,
                                    int jm = 3) {
  int ab[4], bb[2][2];
  a_bases<NP, AC>(L, ab);
  b_bases<NP, BC>(L, bb);
  c.zero();
  if (!jm) return;
  for (int kc = 0; kc < kch; ++kc) {
    double ar[4], ai[4];
    load_a<NP, AC>(A, ab, kc * 8, ar, ai);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (!((jm >> j) & 1)) continue;
      double br[2], bi[2];
      load_b<NP, BC>(B, bb[j], kc * 8, br, bi);
      cmma(c.re[j], c.im[j], ar, ai, br, bi);
    }
  }
}
// c1 = A1 B, c2 = A2 B.
template <int NP>
__device__ __forceinline__ void cmm2b(CAcc& c1, CAcc& c2, const double2* A1, const double2* A2, const double2* B,
                                      int kch, const Lane& L, int jm = 3) {
  int ab[4], bb[2][2];
  a_bases<NP, false>(L, ab);
  b_bases<NP, false>(L, bb);
  c1.zero();
  c2.zero();
  if (!jm) return;
  for (int kc = 0; kc < kch; ++kc) {
    double a1r[4], a1i[4], a2r[4], a2i[4];
    load_a<NP, false>(A1, ab, kc * 8, a1r, a1i);
    load_a<NP, false>(A2, ab, kc * 8, a2r, a2i);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (!((jm >> j) & 1)) continue;
      double br[2], bi[2];
      load_b<NP, false>(B, bb[j], kc * 8, br, bi);
      cmma(c1.re[j], c1.im[j], a1r, a1i, br, bi);
      cmma(c2.re[j], c2.im[j], a2r, a2i, br, bi);
    }
  }
}

// c1 = A B1, c2 = A B2 (the A fragments loaded once; each accumulator sees
// the same tensor instructions as a separate cmm).
template <int NP>
__device__ __forceinline__ void cmm2a(CAcc& c1, CAcc& c2, const double2* A, const double2* B1, const double2* B2,
                                      int kch, const Lane& L, int jm = 3) {
  int ab[4], bb[2][2];
  a_bases<NP, false>(L, ab);
  b_bases<NP, false>(L, bb);
  c1.zero();
  c2.zero();
  if (!jm) return;
  for (int kc = 0; kc < kch; ++kc) {
    double ar[4], ai[4];
    load_a<NP, false>(A, ab, kc * 8, ar, ai);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (!((jm >> j) & 1)) continue;
      double br[2], bi[2];
      load_b<NP, false>(B1, bb[j], kc * 8, br, bi);
      cmma(c1.re[j], c1.im[j], ar, ai, br, bi);
      load_b<NP, false>(B2, bb[j], kc * 8, br, bi);
      cmma(c2.re[j], c2.im[j], ar, ai, br, bi);
    }
  }
}

template <int NP>
__device__ __forceinline__ void store_acc(double2* S, const CAcc& c, const Lane& L, int jm = 3) {
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if ((jm >> j) & 1) S[sidx<NP>(own_r(L, q), own_c(L, j, q))] = c.get(j, q);
}

// Work split of the products between the SM's four sub-partitions (warp
// index mod 4).  With 9 tiles (NP = 48) sub-partition 0 runs the tile
// warps 0, 4 and 8; the right half (j = 1) of tile 8 is computed by a warp
// of sub-partition 3 (kHelper) instead, so the sub-partitions carry 5, 4, 4
// and 5 halves, not 6, 4, 4, 4.  The moved half keeps its arithmetic; in
// the decimation its eps lives in shared memory (lane-private,
// epsx[q * 32 + lane]), owned by the helper.
template <int NP>
struct Split {
  static constexpr bool on = Geo<NP>::NW == 9;
  // The moved half goes to a warp of sub-partition 3: the last warp, which
  // owns no tile when the block has more warps than tiles, else warp 3.
  static constexpr int kHelper = Geo<NP>::NWB > Geo<NP>::NW ? Geo<NP>::NWB - 1 : 3;
  int jt;      // halves of the own tile, 0 for warps without a tile
  int jm;      // halves of the own tile this warp computes in the split products
  bool extra;  // this warp also computes the moved half
  Lane Lx;     // geometry of the moved half's tile (use with j = 1)
  __device__ __forceinline__ explicit Split(const Lane& L) {
    const int w = threadIdx.x >> 5;
    jt = w < Geo<NP>::NW ? 3 : 0;
    jm = (on && w == Geo<NP>::NW - 1) ? 1 : jt;
    extra = on && w == kHelper;
    Lx = L;  // the last tile (NW - 1) of the T x T grid
    Lx.m0 = ((Geo<NP>::NW - 1) / Geo<NP>::T) * 16;
    Lx.n0 = ((Geo<NP>::NW - 1) % Geo<NP>::T) * 16;
  }
};

// Global nr x nc row-major matrix -> padded shared buffer (zeros outside).
template <int NP>
__device__ __forceinline__ void load_mat(double2* S, const double2* __restrict__ G, int nr, int nc) {
  for (int idx = threadIdx.x; idx < NP * NP; idx += Geo<NP>::NTH) {
    const int r = idx / NP, c = idx - r * NP;
    S[sidx<NP>(r, c)] = (r < nr && c < nc) ? G[(long long)r * nc + c] : make_double2(0.0, 0.0);
  }
}

// 1 / (a + ib) by Smith's algorithm (R. L. Smith, CACM 5(8), 1962).
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

// ---------------------------------------------------------- Gauss-Jordan --
// Shared bookkeeping of the blocked Gauss-Jordan inversion (the panel itself
// lives in a caller-provided free matrix buffer).
struct GJShared {
  int* sig;       // logical -> physical row within the current panel
  int* siginv;    // physical -> logical
  int* pivlog;    // pivlog[k]: logical row interchanged with row k at step k
  int* cmap;      // cmap[c] = t_k(...t_0(c)) over the steps done so far
  int* cmapinv;   // its inverse
  unsigned* key;  // [8][NWB] each warp's pivot key of each panel column
};
template <int NP>
__host__ __device__ constexpr int gj_shared_bytes() { return 5 * NP * 4 + 8 * Geo<NP>::NWB * 4; }
template <int NP>
__device__ __forceinline__ GJShared carve_gj(unsigned char* base) {
  GJShared g;
  g.sig = reinterpret_cast<int*>(base);
  g.siginv = g.sig + NP;
  g.pivlog = g.siginv + NP;
  g.cmap = g.pivlog + NP;
  g.cmapinv = g.cmap + NP;
  g.key = reinterpret_cast<unsigned*>(g.cmapinv + NP);
  return g;
}
// Panel element (row r, column c < 8), rows of 8 with the row swizzle.
__device__ __forceinline__ int pidx(int r, int c) { return r * 8 + (c ^ swz(r)); }

// Pivot key of a candidate entry: top bits of max(|re|, |im|) with the row
// index (< 64) in the low 6 bits, so the unsigned maximum over a column picks
// the largest entry up to a relative 2^-14, ties to the lowest row.
__device__ __forceinline__ unsigned pivot_key(double2 v, int r) {
  const unsigned ha = (unsigned)__double2hiint(v.x) & 0x7fffffffu;
  const unsigned hb = (unsigned)__double2hiint(v.y) & 0x7fffffffu;
  const unsigned hm = ha > hb ? ha : hb;
  return (hm & ~63u) | (unsigned)(63 - r);
}

// Rank-8 update of one 16 x 16 tile (halves jm) by the factored panel
// W = lambda P held in P (rows by physical row, sig: logical -> physical):
//     next(r, Q) = [r not a pivot row] cur(sig r, Q) + P(sig r, :) W(sig(pivot rows), Q)
//     next(r, panel) = P(sig r, :)
// with P = W / lambda.  The half holding the panel's columns only stores
// P(sig r, :) (its rank-8 sum would be discarded).
template <int NP>
__device__ __forceinline__ void rank8_tile(const double2* cur, double2* nxt, const double2* P, const int* sig,
                                           double2 lam, int k0, int jmax, const Lane& T, int jm) {
  const int ph = ((k0 >> 4) == (T.n0 >> 4)) ? ((k0 >> 3) & 1) : -1;  // the panel's half of this tile
  const double2 il = crecip_smith(lam);
  int srow[2];
  bool inpanel[2];
#pragma unroll
  for (int ri = 0; ri < 2; ++ri) {
    const int r = T.m0 + T.g + 8 * ri;
    srow[ri] = sig[r];
    inpanel[ri] = r >= k0 && r < k0 + jmax;
  }
  double ar[4], ai[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double2 v = cmul(P[pidx(srow[q & 1], T.t + 4 * (q >> 1))], il);
    ar[q] = v.x;
    ai[q] = v.y;
  }
  const int kk0 = T.t, kk1 = T.t + 4;
  const int pr0 = kk0 < jmax ? sig[k0 + kk0] : 0, pr1 = kk1 < jmax ? sig[k0 + kk1] : 0;
#pragma unroll
  for (int j2 = 0; j2 < 2; ++j2) {
    if (!((jm >> j2) & 1)) continue;
    if (j2 == ph) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int cc = own_c(T, j2, q);
        nxt[sidx<NP>(own_r(T, q), cc)] = cmul(P[pidx(srow[q >> 1], cc - k0)], il);
      }
      continue;
    }
    double cr[4], ci[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double2 v = cur[sidx<NP>(srow[q >> 1], own_c(T, j2, q))];
      cr[q] = inpanel[q >> 1] ? 0.0 : v.x;
      ci[q] = inpanel[q >> 1] ? 0.0 : v.y;
    }
    const int cc = T.n0 + 8 * j2 + T.g;
    const double2 v0 = cur[sidx<NP>(pr0, cc)], v1 = cur[sidx<NP>(pr1, cc)];
    double br[2], bi[2];
    br[0] = kk0 < jmax ? v0.x : 0.0;
    bi[0] = kk0 < jmax ? v0.y : 0.0;
    br[1] = kk1 < jmax ? v1.x : 0.0;
    bi[1] = kk1 < jmax ? v1.y : 0.0;
    cmma(cr, ci, ar, ai, br, bi);
#pragma unroll
    for (int q = 0; q < 4; ++q) nxt[sidx<NP>(own_r(T, q), own_c(T, j2, q))] = make_double2(cr[q], ci[q]);
  }
}

// Rank-8 work split: at NP = 48 (9 tile warps in 12) the right half of tile
// 8 moves from sub-partition 0 to warp 10 (sub-partition 2), which owns no
// tile and does no Gauss-Jordan bookkeeping.
template <int NP>
struct R8Split {
  static constexpr bool on = Geo<NP>::NW == 9 && Geo<NP>::NWB >= 11;
  int jm;      // halves to compute: of the own tile, or the moved half (2)
  bool extra;  // this warp takes the moved half
  Lane Lx;     // the moved half's tile (use with j = 1)
  __device__ __forceinline__ explicit R8Split(const Lane& L) {
    const int w = threadIdx.x >> 5;
    extra = on && w == Geo<NP>::NW + 1;
    jm = extra ? 2 : ((on && w == Geo<NP>::NW - 1) ? 1 : 3);
    Lx = L;
    Lx.m0 = ((Geo<NP>::NW - 1) / Geo<NP>::T) * 16;
    Lx.n0 = ((Geo<NP>::NW - 1) % Geo<NP>::T) * 16;
  }
};

// Inverse of the leading n x n block of X (padding = identity, n <= NP <= 64)
// by blocked Gauss-Jordan elimination with partial pivoting.  Y is the second
// matrix buffer and Z (at least 2 NP x 8 complex) holds the panel; *out
// receives the buffer holding the inverse (X or Y).
//
// Columns are processed in panels of 8.  The n x 8 panel is factored by the
// whole block with one barrier per column and no division: the panel is kept
// as W = lambda P (P the textbook Gauss-Jordan panel, lambda a complex
// scalar) and, with p the pivot and s a power of two bringing p near 1,
//     new(r, c) = (p s) a' - (s b') m,   lambda <- lambda p s
//     a' = 0 if r is the pivot row or c the pivot column, else W(r, c)
//     b' = -lambda for the pivot row, else W(r, j)
//     m  =  lambda for the pivot column, else W(pivot row, c)
// (expanding W = lambda P gives the textbook update times the new lambda;
// |p s| lies in [1, 2.83]).  Pivot search is looked ahead: the threads that
// write column j+1 of the panel reduce its pivot keys (see pivot_key) over
// the rows not yet used as pivots into key[j+1] before the barrier, so step
// j+1 starts from one shared load; the key's exponent bits give s.  The row
// interchanges are kept as a permutation (sig).  Then every warp applies the
// panel to the whole matrix as a rank-8 product on the FP64 tensor path,
// writing the next buffer in the new row order:
//     next(r, Q) = [r not a pivot row] W(sig r, Q) + P(sig r, :) W(sig(pivot rows), Q)
//     next(r, panel) = P(sig r, :),   P = W / lambda
// The interchanges are undone at the end as column interchanges (column c of
// the inverse is column t_{n-1}(...t_0(c)) of the eliminated matrix,
// t_k = (k pivlog_k)) in one gather.  Returns kOk, kSingular (all candidates
// zero or below 2^-1022) or kNonFinite identically in every thread.
template <int NP>
__device__ int gj_invert(double2* X, double2* Y, double2* Z, int n, const Lane& L, const GJShared& sh,
                         double2** out) {
  static_assert(NP <= 64, "pivot keys carry a 6-bit row index");
  constexpr int NTH = Geo<NP>::NTH;
  const bool tw = (int)(threadIdx.x >> 5) < Geo<NP>::NW;  // this warp owns a tile
  constexpr int PE = NP * 8;                  // panel elements
  constexpr int PPT = (PE + NTH - 1) / NTH;   // panel elements per thread
  const int tid = threadIdx.x, lane = tid & 31;
  const R8Split<NP> r8(L);
  double2* cur = X;
  double2* nxt = Y;
  int rows[2], rbase[2], rsw[2];
#pragma unroll
  for (int ri = 0; ri < 2; ++ri) {
    rows[ri] = L.m0 + L.g + 8 * ri;
    rbase[ri] = rows[ri] * NP;
    rsw[ri] = swz(rows[ri]);
  }
  int cols[4];
#pragma unroll
  for (int ci = 0; ci < 4; ++ci) cols[ci] = L.n0 + 8 * (ci >> 1) + 2 * L.t + (ci & 1);
  for (int c = tid; c < NP; c += NTH) {  // visible after the first panel's barrier
    sh.cmap[c] = c;
    sh.cmapinv[c] = c;
  }
  // Panel elements owned by this thread: element e = tid + q NTH.  A partly
  // filled last slot (n = 48: 96 elements) goes to warps 1, 2, 3 rather
  // than 0, 1, 2, so that each of the SM's four sub-partitions (warp index
  // mod 4) carries the same number of slots.
  int pr_[PPT], pc_[PPT];
  bool pin[PPT];
#pragma unroll
  for (int q = 0; q < PPT; ++q) {
    const bool partial = (q + 1) * NTH > PE;
    const int e = partial ? tid - 32 + q * NTH : tid + q * NTH;
    pin[q] = partial ? (tid >= 32 && e < PE) : true;
    pr_[q] = pin[q] ? (e >> 3) : 0;
    pc_[q] = (pin[q] ? e : 0) & 7;
  }

  for (int k0 = 0; k0 < n; k0 += 8) {
    const int jmax = (n - k0) < 8 ? (n - k0) : 8;
    double2* P = Z;
    double2* Pn = Z + PE;
    bool used[PPT];
    // Each thread also keeps its own panel elements in registers (av), so a
    // column step reads from shared memory only what other threads wrote:
    // its row's entry of the pivot column and the pivot row.
    double2 av[PPT];
    // ---- load the panel, reset the bookkeeping, keys of panel column 0 ----
    unsigned key0 = 0u;
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
      const int r = pr_[q], c = pc_[q];
      used[q] = false;
      av[q] = make_double2(0.0, 0.0);
      if (pin[q]) {
        const double2 v = cur[sidx<NP>(r, k0 + c)];
        P[pidx(r, c)] = v;
        av[q] = v;
        if (c == 0 && r >= k0 && r < n) key0 = max(key0, pivot_key(v, r));
      }
    }
    for (int r = tid; r < NP; r += NTH) {
      sh.sig[r] = r;
      sh.siginv[r] = r;
    }
    // Each warp posts its key in its own slot (no shared atomics); after the
    // barrier lane i of every warp reads slot i and the warp takes the max.
    key0 = __reduce_max_sync(0xffffffffu, key0);
    if (lane == 0) sh.key[tid >> 5] = key0;
    __syncthreads();
    double2 lam = make_double2(1.0, 0.0);
    // ---- factor the panel, one barrier per column ----
    for (int j = 0; j < jmax; ++j) {
      // The own rows' pivot-column entries do not depend on the pivot: load
      // them with the key.  The key slots are read one lane per slot and
      // reduced in the warp (one shared-memory wavefront per warp).
      double2 mv[PPT], fv[PPT];
#pragma unroll
      for (int q = 0; q < PPT; ++q) fv[q] = P[pidx(pr_[q], j)];
      const unsigned key =
          __reduce_max_sync(0xffffffffu, lane < Geo<NP>::NWB ? sh.key[j * Geo<NP>::NWB + lane] : 0u);
      if ((key >> 20) >= 0x7ffu) return kNonFinite;
      if ((key >> 6) == 0u) return kSingular;
      const int pr = 63 - (int)(key & 63u);
      const int ex = (int)(key >> 20);
      const double sc = (ex != 0 && ex < 2046) ? __hiloint2double((2046 - ex) << 20, 0) : 1.0;
      // Row interchange bookkeeping by the last warp (at n = 48 a warp with
      // no product tile): its two loads go out with the pivot row's, its
      // stores after the element update.
      const bool bk = (tid == NTH - 32);
      const int k = k0 + j;
      int bl = 0, pa = 0;
      if (bk) {
        bl = sh.siginv[pr];
        pa = sh.sig[k];
      }
      const double2 piv = P[pidx(pr, j)];
#pragma unroll
      for (int q = 0; q < PPT; ++q) mv[q] = P[pidx(pr, pc_[q])];
      const double2 ps = make_double2(piv.x * sc, piv.y * sc);
      unsigned nk = 0u;
#pragma unroll
      for (int q = 0; q < PPT; ++q) {
        // Slots past the panel are whole warps (PE and NTH are multiples of
        // 32), so this skips their arithmetic without divergence.
        if (!pin[q]) continue;
        const int r = pr_[q], c = pc_[q];
        const bool isp = (r == pr);
        used[q] = used[q] || isp;
        const double2 bb = isp ? cneg(lam) : fv[q];
        const double2 b = make_double2(bb.x * sc, bb.y * sc);
        const double2 m = (c == j) ? lam : mv[q];
        double2 v = cneg(cmul(b, m));
        if (!isp && c != j) cfma(v, ps, av[q]);
        Pn[pidx(r, c)] = v;
        av[q] = v;
        if (c == j + 1 && !used[q] && r >= k0 && r < n) nk = max(nk, pivot_key(v, r));
      }
      lam = cmul(lam, ps);
      if (j + 1 < jmax) {
        nk = __reduce_max_sync(0xffffffffu, nk);
        if (lane == 0) sh.key[(j + 1) * Geo<NP>::NWB + (tid >> 5)] = nk;
      }
      if (bk) {
        sh.sig[k] = pr;
        sh.sig[bl] = pa;
        sh.siginv[pr] = k;
        sh.siginv[pa] = bl;
        sh.pivlog[k] = bl;
      }
      __syncthreads();
      double2* t = P;
      P = Pn;
      Pn = t;
    }
    // ---- rank-8 update of the whole matrix ----
    // The tile warps take their tiles; at NP = 48 the right half of the last
    // tile goes to a warp without a tile on another sub-partition (kR8Helper),
    // so that sub-partition 0 carries 5 halves instead of 6.
    if (tw || r8.extra) rank8_tile<NP>(cur, nxt, P, sh.sig, lam, k0, jmax, r8.extra ? r8.Lx : L, r8.jm);
    // The panel's interchanges t_k = (k pivlog_k) applied to the column map,
    // by the bookkeeping thread (at n = 48 a warp without rank-8 work):
    // cmap <- t_k o cmap swaps the two entries holding the values k and b.
    if (tid == NTH - 32) {
      for (int j = 0; j < jmax; ++j) {
        const int k = k0 + j, b2 = sh.pivlog[k];
        if (b2 != k) {
          const int c1 = sh.cmapinv[k], c2 = sh.cmapinv[b2];
          sh.cmap[c1] = b2;
          sh.cmap[c2] = k;
          sh.cmapinv[k] = c2;
          sh.cmapinv[b2] = c1;
        }
      }
    }
    __syncthreads();
    double2* t = cur;
    cur = nxt;
    nxt = t;
  }
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const int ri = (e & 3) >> 1, ci = (e >> 2) * 2 + (e & 1);
    if (tw) nxt[rbase[ri] + (cols[ci] ^ rsw[ri])] = cur[rbase[ri] + (sh.cmap[cols[ci]] ^ rsw[ri])];
  }
  __syncthreads();
  *out = nxt;
  return kOk;
}

// Bytes after the matrix buffers: Gauss-Jordan scratch, then reduction slots.
template <int NP>
__host__ __device__ constexpr int tail_bytes() { return gj_shared_bytes<NP>() + 40 * 8; }
template <int NP>
__device__ __forceinline__ double* carve_red(double2* tail) {
  return reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(tail) + gj_shared_bytes<NP>());
}

// ------------------------------------------------------------ Sancho-Rubio --
// Shared buffers: alpha, beta, g (inverse, then the next alpha), alpha g,
// beta g, eps_s.  eps lives in registers.  Every thread reads and writes
// only its own elements of eps and eps_s, so those need no barriers.
template <int NP>
constexpr int sr_buffers() { return 6; }

template <int NP>
__global__ void __launch_bounds__(Geo<NP>::NTH, 1) sr_f64_kernel(SrArgs a) {
  using G = Geo<NP>;
  constexpr int MAT = G::MAT;
  extern __shared__ __align__(16) unsigned char smraw[];
  // Roles rotate between iterations: pa = alpha, pb = beta, f0..f2 free,
  // pes = eps_s (owner-only access).
  double2* pa = reinterpret_cast<double2*>(smraw);
  double2* pb = pa + MAT;
  double2* f0 = pb + MAT;
  double2* f1 = f0 + MAT;
  double2* f2 = f1 + MAT;
  double2* pes = f2 + MAT;
  const GJShared gsh = carve_gj<NP>(reinterpret_cast<unsigned char*>(pes + MAT));
  double* red = carve_red<NP>(pes + MAT);
  double2* epsx = reinterpret_cast<double2*>(red + 40);  // eps of the moved half (Split)

  const int p = blockIdx.x;
  if (p >= a.batch) return;
  const int n = a.n;
  const int kch = (n + 7) >> 3;
  const int tid = threadIdx.x;
  const Lane L = lane_geo<NP>();
  const long long kset = a.kidx ? (long long)a.kidx[p] : 0;
  const double2* h00 = a.h00 + kset * a.lead_stride;
  const double2* h01 = a.h01 + kset * a.lead_stride;
  const double2* h10 = a.h10 ? a.h10 + kset * a.lead_stride : nullptr;
  const double w = a.omega[p];
  const double2 z = z_of(w, a.eta[p]);

  const Split<NP> sp(L);
  const int lane = tid & 31;
  double2 eps[8];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = own_r(L, q), c = own_c(L, j, q);
      const double2 e = (r < n && c < n) ? h00[r * n + c] : make_double2(0.0, 0.0);
      eps[j * 4 + q] = e;
      if ((sp.jm >> j) & 1) pes[sidx<NP>(r, c)] = e;
    }
  if (sp.extra) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = own_r(sp.Lx, q), c = own_c(sp.Lx, 1, q);
      const double2 e = (r < n && c < n) ? h00[r * n + c] : make_double2(0.0, 0.0);
      epsx[q * 32 + lane] = e;
      pes[sidx<NP>(r, c)] = e;
    }
  }
  for (int idx = tid; idx < NP * NP; idx += G::NTH) {
    const int r = idx / NP, c = idx - r * NP;
    const bool in = r < n && c < n;
    pa[sidx<NP>(r, c)] = in ? h01[r * n + c] : make_double2(0.0, 0.0);
    pb[sidx<NP>(r, c)] = in ? (h10 ? h10[r * n + c] : cconj(h01[c * n + r])) : make_double2(0.0, 0.0);
  }

  int status = kOk;
  int it = 0;
  const double tol2 = a.tol * a.tol;
  CAcc c1, c2;
  bool converged = false;
  double2* pg = nullptr;
  for (it = 1; it <= a.maxiter; ++it) {
    // M = z - eps (identity in the padding) into f0, inverted via f1.
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (!((sp.jm >> j) & 1)) continue;
        const int r = own_r(L, q), c = own_c(L, j, q);
        double2 v;
        if (r < n && c < n) v = (r == c) ? csub(z, eps[j * 4 + q]) : cneg(eps[j * 4 + q]);
        else v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        f0[sidx<NP>(r, c)] = v;
      }
    if (sp.extra) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = own_r(sp.Lx, q), c = own_c(sp.Lx, 1, q);
        const double2 e = epsx[q * 32 + lane];
        double2 v;
        if (r < n && c < n) v = (r == c) ? csub(z, e) : cneg(e);
        else v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        f0[sidx<NP>(r, c)] = v;
      }
    }
    __syncthreads();
    status = gj_invert<NP>(f0, f1, f2, n, L, gsh, &pg);
    if (status != kOk) break;
    double2* pag = (pg == f0) ? f1 : f0;  // the inversion's other buffer
    double2* pbg = f2;
    // alpha g, beta g
    cmm2b<NP>(c1, c2, pa, pb, pg, kch, L, sp.jm);
    store_acc<NP>(pag, c1, L, sp.jm);
    store_acc<NP>(pbg, c2, L, sp.jm);
    if (sp.extra) {
      cmm2b<NP>(c1, c2, pa, pb, pg, kch, sp.Lx, 2);
      store_acc<NP>(pag, c1, sp.Lx, 2);
      store_acc<NP>(pbg, c2, sp.Lx, 2);
    }
    __syncthreads();
    // Pass A, shared A = alpha g: eps_s += (alpha g) beta, eps += (alpha g) beta,
    // alpha' = (alpha g) alpha into the free g buffer.
    // Pass B, shared A = beta g: eps += (beta g) alpha, beta' = (beta g) beta
    // (stored after the barrier that ends every read of alpha and beta).
    int bad = 0;
    double e2 = 0.0;
    cmm2a<NP>(c1, c2, pag, pb, pa, kch, L, sp.jm);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (!((sp.jm >> j) & 1)) continue;
        const int e = sidx<NP>(own_r(L, q), own_c(L, j, q));
        const double2 es = cadd(pes[e], c1.get(j, q));
        pes[e] = es;
        eps[j * 4 + q] = cadd(eps[j * 4 + q], c1.get(j, q));
        bad |= !cfinite(es);
        bad |= !cfinite(c2.get(j, q));
        e2 = fmax(e2, cabs2(c2.get(j, q)));
      }
    store_acc<NP>(pg, c2, L, sp.jm);
    if (sp.extra) {
      cmm2a<NP>(c1, c2, pag, pb, pa, kch, sp.Lx, 2);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = sidx<NP>(own_r(sp.Lx, q), own_c(sp.Lx, 1, q));
        const double2 es = cadd(pes[e], c1.get(1, q));
        pes[e] = es;
        epsx[q * 32 + lane] = cadd(epsx[q * 32 + lane], c1.get(1, q));
        bad |= !cfinite(es);
        bad |= !cfinite(c2.get(1, q));
        e2 = fmax(e2, cabs2(c2.get(1, q)));
      }
      store_acc<NP>(pg, c2, sp.Lx, 2);
    }
    cmm2a<NP>(c1, c2, pbg, pa, pb, kch, L, sp.jm);
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (!((sp.jm >> j) & 1)) continue;
        eps[j * 4 + q] = cadd(eps[j * 4 + q], c1.get(j, q));
        bad |= !cfinite(eps[j * 4 + q]);
        bad |= !cfinite(c2.get(j, q));
        e2 = fmax(e2, cabs2(c2.get(j, q)));
      }
    if (sp.extra) {  // the helper owns no tile, so c2 is free for the moved half's beta'
      cmm2a<NP>(c1, c2, pbg, pa, pb, kch, sp.Lx, 2);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double2 e = cadd(epsx[q * 32 + lane], c1.get(1, q));
        epsx[q * 32 + lane] = e;
        bad |= !cfinite(e);
        bad |= !cfinite(c2.get(1, q));
        e2 = fmax(e2, cabs2(c2.get(1, q)));
      }
    }
    __syncthreads();  // every read of alpha and beta is done
    store_acc<NP>(pb, c2, L, sp.jm);
    if (sp.extra) store_acc<NP>(pb, c2, sp.Lx, 2);
    f0 = pa;  // old alpha buffer is free
    f1 = pag;
    f2 = pbg;
    pa = pg;
    if (block_any(bad)) {
      status = sr_failure_status(it, n, h00, h01, h10, z);
      break;
    }
    const double emax = block_max(e2, red);
    if (emax < tol2) { converged = true; break; }
  }
  if (status == kOk && !converged) {
    status = kMaxIter;
    it = a.maxiter;
  }
  if (status == kOk) {
    // every element of eps_s is in shared memory: each thread builds its own tile
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (!((sp.jt >> j) & 1)) continue;
        const int r = own_r(L, q), c = own_c(L, j, q);
        const double2 es = pes[sidx<NP>(r, c)];
        double2 v;
        if (r < n && c < n) v = (r == c) ? csub(z, es) : cneg(es);
        else v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        f0[sidx<NP>(r, c)] = v;
      }
    __syncthreads();
    status = gj_invert<NP>(f0, f1, f2, n, L, gsh, &pg);
  }
  if (status == kOk) {
    if (a.g_out) {
      double2* go = a.g_out + (long long)p * n * n;
      for (int idx = tid; idx < n * n; idx += G::NTH) {
        const int r = idx / n, c = idx - r * n;
        go[idx] = pg[sidx<NP>(r, c)];
      }
    }
    if (a.dos_out) {
      // (omega/pi) Re Tr[i (g - g^H)] = (omega/pi) sum_j (-2 Im g_jj)
      double t = 0.0;
      for (int j = tid; j < n; j += G::NTH) t += -2.0 * pg[sidx<NP>(j, j)].y;
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
}

// ---------------------------------------------------------------- RGF sweep --
// Shared buffers: pg (left-connected g_l) and pc (coupling / scratch) swap
// roles with the inversion; bW = g_{l-1} C, bU = G_{0,l-1} C, bG0 = G_{0,l}.
template <int NP>
__global__ void __launch_bounds__(Geo<NP>::NTH, 1) rgf_f64_kernel(RgfArgs a) {
  using G = Geo<NP>;
  constexpr int MAT = G::MAT;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* const b0 = reinterpret_cast<double2*>(smraw);
  double2* const b1 = b0 + MAT;
  double2* const bW = b1 + MAT;
  double2* const bU = bW + MAT;
  double2* const bG0 = bU + MAT;
  double2* const bC = bG0 + MAT;  // the coupling block C of the current layer
  const GJShared gsh = carve_gj<NP>(reinterpret_cast<unsigned char*>(bC + MAT));
  double* red = carve_red<NP>(bC + MAT);
  __shared__ int s_point;

  const int n = a.n, L = a.L;
  const int kch = (n + 7) >> 3;
  const int tid = threadIdx.x;
  const Lane Ln = lane_geo<NP>();
  // Per-layer products split between sub-partitions as in the decimation
  // (Split); the once-per-point self-energies and trace keep whole tiles, so
  // the trace's block sum adds the same per-thread terms as before.
  const Split<NP> sp(Ln);
  double2* sigL = a.sigma_ws + (long long)blockIdx.x * 2 * n * n;
  double2* sigR = sigL + (long long)n * n;
  CAcc c1, c2;

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
    double2* pg = b0;
    double2* pc = b1;

    // Contact self-energies Sigma = V g V^H into this block's scratch.
    for (int side = 0; side < 2; ++side) {
      const int nl = side ? a.nr : a.nl;
      const int lch = (nl + 7) >> 3;
      const double2* V = side ? a.VR + k * a.vr_ks : a.VL + k * a.vl_ks;
      const double2* g = side ? a.gR + (long long)p * a.gr_ps : a.gL + (long long)p * a.gl_ps;
      double2* S = side ? sigR : sigL;
      load_mat<NP>(pc, V, n, nl);
      load_mat<NP>(bW, g, nl, nl);
      __syncthreads();
      cmm<NP, false, false>(c1, pc, bW, lch, Ln, sp.jt);
      store_acc<NP>(bU, c1, Ln, sp.jt);
      __syncthreads();
      cmm<NP, false, true>(c1, bU, pc, lch, Ln, sp.jt);
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = own_r(Ln, q), c = own_c(Ln, j, q);
          if (((sp.jt >> j) & 1) && r < n && c < n) S[r * n + c] = c1.get(j, q);
        }
      __syncthreads();
    }

    // Layer 0: g_0 = (z - D_0 - Sigma_L [- Sigma_R when L == 1])^-1 = G_{0,0}.
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (!((sp.jt >> j) & 1)) continue;
        const int r = own_r(Ln, q), c = own_c(Ln, j, q);
        double2 v;
        if (r < n && c < n) {
          v = csub(cneg(D[r * n + c]), sigL[r * n + c]);
          if (L == 1) v = csub(v, sigR[r * n + c]);
          if (r == c) v = cadd(v, z);
        } else {
          v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        }
        pg[sidx<NP>(r, c)] = v;
      }
    __syncthreads();
    double2* inv = nullptr;
    int status = gj_invert<NP>(pg, pc, bW, n, Ln, gsh, &inv);
    if (status == kOk) {
      pc = (inv == pg) ? pc : pg;
      pg = inv;
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (!((sp.jt >> j) & 1)) continue;
          const int e = sidx<NP>(own_r(Ln, q), own_c(Ln, j, q));
          bG0[e] = pg[e];
        }
      for (int l = 1; l < L && status == kOk; ++l) {
        // identical layers (layer stride 0) share one C: load it once per point
        if (l == 1 || a.c_ls != 0) {
          load_mat<NP>(bC, C + (long long)(l - 1) * a.c_ls, n, n);
          __syncthreads();
        }
        // W = g_{l-1} C, U = G_{0,l-1} C
        cmm2b<NP>(c1, c2, pg, bG0, bC, kch, Ln, sp.jm);
        store_acc<NP>(bW, c1, Ln, sp.jm);
        store_acc<NP>(bU, c2, Ln, sp.jm);
        if (sp.extra) {
          cmm2b<NP>(c1, c2, pg, bG0, bC, kch, sp.Lx, 2);
          store_acc<NP>(bW, c1, sp.Lx, 2);
          store_acc<NP>(bU, c2, sp.Lx, 2);
        }
        __syncthreads();
        // M = z - D_l - C^H W [- Sigma_R on the last layer] into the old g buffer
        const double2* Dl = D + (long long)l * a.d_ls;
        const bool last = (l == L - 1);
        auto form_m = [&](const Lane& Lm, int jm) {
          cmm<NP, true, false>(c1, bC, bW, kch, Lm, jm);
#pragma unroll
          for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              if (!((jm >> j) & 1)) continue;
              const int r = own_r(Lm, q), c = own_c(Lm, j, q);
              double2 v;
              if (r < n && c < n) {
                v = csub(cneg(Dl[r * n + c]), c1.get(j, q));
                if (last) v = csub(v, sigR[r * n + c]);
                if (r == c) v = cadd(v, z);
              } else {
                v = make_double2(r == c ? 1.0 : 0.0, 0.0);
              }
              pg[sidx<NP>(r, c)] = v;
            }
        };
        form_m(Ln, sp.jm);
        if (sp.extra) form_m(sp.Lx, 2);
        __syncthreads();
        status = gj_invert<NP>(pg, pc, bW, n, Ln, gsh, &inv);
        if (status != kOk) break;
        pc = (inv == pg) ? pc : pg;
        pg = inv;
        // G_{0,l} = U g_l
        cmm<NP, false, false>(c1, bU, pg, kch, Ln, sp.jm);
        store_acc<NP>(bG0, c1, Ln, sp.jm);
        if (sp.extra) {
          cmm<NP, false, false>(c1, bU, pg, kch, sp.Lx, 2);
          store_acc<NP>(bG0, c1, sp.Lx, 2);
        }
        __syncthreads();
      }
    }
    double tval = 0.0;
    if (status == kOk) {
      // Gamma = i (Sigma - Sigma^H) for both contacts.
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (!((sp.jt >> j) & 1)) continue;
          const int r = own_r(Ln, q), c = own_c(Ln, j, q);
          double2 gl = make_double2(0.0, 0.0), gr = gl;
          if (r < n && c < n) {
            double2 d = csub(sigL[r * n + c], cconj(sigL[c * n + r]));
            gl = make_double2(-d.y, d.x);
            d = csub(sigR[r * n + c], cconj(sigR[c * n + r]));
            gr = make_double2(-d.y, d.x);
          }
          pc[sidx<NP>(r, c)] = gl;
          bW[sidx<NP>(r, c)] = gr;
        }
      __syncthreads();
      cmm<NP, false, false>(c1, pc, bG0, kch, Ln, sp.jt);
      store_acc<NP>(bU, c1, Ln, sp.jt);
      __syncthreads();
      cmm<NP, false, false>(c1, bU, bW, kch, Ln, sp.jt);
      double t = 0.0;
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (!((sp.jt >> j) & 1)) continue;
          const double2 g = bG0[sidx<NP>(own_r(Ln, q), own_c(Ln, j, q))];
          t += c1.re[j][q] * g.x + c1.im[j][q] * g.y;
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

// ------------------------------------------------------------ 1 x 1 blocks --
__global__ void sr_scalar_kernel(SrArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.batch) return;
  const long long k = a.kidx ? (long long)a.kidx[p] : 0;
  const double2 h00 = a.h00[k * a.lead_stride];
  const double2 h01 = a.h01[k * a.lead_stride];
  const double2 h10 = a.h10 ? a.h10[k * a.lead_stride] : cconj(h01);
  const double w = a.omega[p];
  const double2 z = z_of(w, a.eta[p]);
  double2 al = h01, be = h10, e = h00, es = h00;
  int status = kOk, it;
  bool conv = false;
  const double tol2 = a.tol * a.tol;
  for (it = 1; it <= a.maxiter; ++it) {
    const double2 m = csub(z, e);
    if (m.x == 0.0 && m.y == 0.0) { status = kSingular; break; }
    const double2 g = crecip(m);
    const double2 ag = cmul(al, g), bg = cmul(be, g);
    const double2 agb = cmul(ag, be), bga = cmul(bg, al);
    es = cadd(es, agb);
    e = cadd(cadd(e, agb), bga);
    al = cmul(ag, al);
    be = cmul(bg, be);
    if (!cfinite(es) || !cfinite(e) || !cfinite(al) || !cfinite(be)) {
      // as sr_failure_status, for one thread's 1 x 1 blocks
      const bool quiet = it == 1 && !(cfinite(h00) && cfinite(h01) && cfinite(h10) && cfinite(z));
      status = quiet ? kNonFinite : kUnstable;
      break;
    }
    if (fmax(cabs2(al), cabs2(be)) < tol2) { conv = true; break; }
  }
  if (status == kOk && !conv) { status = kMaxIter; it = a.maxiter; }
  double2 gs = make_double2(0.0, 0.0);
  if (status == kOk) {
    const double2 m = csub(z, es);
    if (m.x == 0.0 && m.y == 0.0) status = kSingular;
    else gs = crecip(m);
  }
  if (status == kOk && a.g_out) a.g_out[p] = gs;
  if (a.dos_out)
    a.dos_out[p] = (status == kOk) ? (w / 3.141592653589793238462643383279502884) * (-2.0 * gs.y)
                                   : __longlong_as_double(0x7ff8000000000000ULL);
  if (a.iters_out) a.iters_out[p] = it;
  if (a.status_out) a.status_out[p] = status;
}

__global__ void rgf_scalar_kernel(RgfArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.batch) return;
  const int lst = a.lead_status ? a.lead_status[p] : 0;
  if (lst != kOk) {
    a.T_out[p] = __longlong_as_double(0x7ff8000000000000ULL);
    if (a.status_out) a.status_out[p] = lst;
    return;
  }
  const long long k = a.kidx ? (long long)a.kidx[p] : 0;
  const double2 z = z_of(a.omega[p], a.eta_dev[p]);
  const double2 vl = a.VL[k * a.vl_ks], vr = a.VR[k * a.vr_ks];
  const double2 sl = cmul(cmul(vl, a.gL[(long long)p * a.gl_ps]), cconj(vl));
  const double2 sr = cmul(cmul(vr, a.gR[(long long)p * a.gr_ps]), cconj(vr));
  const double2* D = a.D + k * a.d_ks;
  const double2* C = a.C + k * a.c_ks;
  const int L = a.L;
  int status = kOk;
  double2 m = csub(csub(z, D[0]), sl);
  if (L == 1) m = csub(m, sr);
  double2 g = make_double2(0.0, 0.0), g0 = g;
  if (m.x == 0.0 && m.y == 0.0) status = kSingular;
  else { g = crecip(m); g0 = g; }
  for (int l = 1; l < L && status == kOk; ++l) {
    const double2 c = C[(long long)(l - 1) * a.c_ls];
    const double2 w = cmul(g, c);
    const double2 u = cmul(g0, c);
    m = csub(csub(z, D[(long long)l * a.d_ls]), cmul(cconj(c), w));
    if (l == L - 1) m = csub(m, sr);
    if (m.x == 0.0 && m.y == 0.0) { status = kSingular; break; }
    g = crecip(m);
    g0 = cmul(u, g);
  }
  double t = 0.0;
  if (status == kOk) {
    // Gamma = i (S - S^*) = -2 Im(S) for 1 x 1 blocks
    const double gl = -2.0 * sl.y, gr = -2.0 * sr.y;
    t = gl * gr * cabs2(g0);
    if (!isfinite(t)) status = kNonFinite;
  }
  a.T_out[p] = (status == kOk) ? t : __longlong_as_double(0x7ff8000000000000ULL);
  if (a.status_out) a.status_out[p] = status;
}

// ------------------------------------------------------------- k-avg, kappa --
// tbar[w] = mean_k T[w, k] over points laid out omega-major (index w*K + k).
__global__ void kavg_kernel(const double* __restrict__ T, int W, int K, double* __restrict__ tbar) {
  const int w = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= W) return;
  double s = 0.0;
  for (int k = lane; k < K; k += 32) s += T[(long long)w * K + k];
  s = warp_sum(s);
  if (lane == 0) tbar[w] = s / (double)K;
}

// k moments <T> and <T^2> of an omega-major [W][K] table, one warp per omega
// (the moments of negfpy workflows/ifc_bulk.py:1690-1784).
__global__ void kmoments_kernel(const double* __restrict__ T, int W, int K, double* __restrict__ t1,
                                double* __restrict__ t2) {
  const int w = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= W) return;
  double s = 0.0, q = 0.0;
  for (int k = lane; k < K; k += 32) {
    const double v = T[(long long)w * K + k];
    s += v;
    q += v * v;
  }
  s = warp_sum(s);
  q = warp_sum(q);
  if (lane == 0) {
    t1[w] = s / (double)K;
    t2[w] = q / (double)K;
  }
}

// Heat-current cumulants from transmission moments (negfpy
// core/fcs.py:48-150), one block:
//   C1 = (1/2pi) trapz(<T> (A_L - A_R), w),
//   C2 = (1/2pi) trapz(<T> (B_L + B_R) + (<T> + <T^2>) (A_L - A_R)^2, w),
//   A = kB T phi1(x), B = (kB T)^2 phi2(x), x = hbar w / (kB T),
//   phi1 = x / expm1(x), phi2 = x^2 e^x / expm1(x)^2, with negfpy's series for
//   |x| < 1e-6 and 0 from x = 700 on.
__device__ __forceinline__ double fcs_phi1(double x) {
  if (fabs(x) < 1e-6) return 1.0 - 0.5 * x + (x * x) / 12.0 - (x * x * x * x) / 720.0;
  if (x < 700.0) return x / expm1(x);
  return 0.0;
}
__device__ __forceinline__ double fcs_phi2(double x) {
  if (fabs(x) < 1e-6) return 1.0 - (x * x) / 12.0 + (x * x * x * x) / 240.0;
  if (x < 700.0) {
    const double em1 = expm1(x);
    return (x * x) * (em1 + 1.0) / (em1 * em1);
  }
  return 0.0;
}
__global__ void fcs_kernel(const double* __restrict__ om, const double* __restrict__ t1, const double* __restrict__ t2,
                           int W, double temp_l, double temp_r, double* __restrict__ out) {
  __shared__ double red[40];
  const double hbar = 1.054571817e-34, kb = 1.380649e-23;
  const double sl = kb * temp_l, sr = kb * temp_r;
  double c1 = 0.0, c2 = 0.0;
  for (int i = threadIdx.x; i < W - 1; i += blockDim.x) {
    double f1[2], f2[2];
    for (int q = 0; q < 2; ++q) {
      const double w = om[i + q];
      const double xl = hbar * w / sl, xr = hbar * w / sr;
      const double ad = __dmul_rn(sl, fcs_phi1(xl)) - __dmul_rn(sr, fcs_phi1(xr));
      const double bs = sl * sl * fcs_phi2(xl) + sr * sr * fcs_phi2(xr);
      const double a = t1[i + q], b = t2[i + q];
      f1[q] = a * ad;
      f2[q] = a * bs + (a + b) * (ad * ad);
    }
    const double dw = om[i + 1] - om[i];
    c1 += dw * (f1[0] + f1[1]) / 2.0;
    c2 += dw * (f2[0] + f2[1]) / 2.0;
  }
  c1 = block_sum(c1, red);
  c2 = block_sum(c2, red);
  if (threadIdx.x == 0) {
    const double pref = 1.0 / (2.0 * 3.141592653589793238462643383279502884);
    out[0] = pref * c1;
    out[1] = pref * c2;
  }
}

// kappa(T) = (1/2pi) trapz(kB tbar(w) x^2 e^-x / (1 - e^-x)^2, w_rad), one
// block per temperature (negfpy workflows/ifc_bulk.py:408-438).
__global__ void kappa_kernel(const double* __restrict__ om, const double* __restrict__ tbar, int W,
                             const double* __restrict__ temps, double unit, double* __restrict__ out) {
  __shared__ double red[40];
  const double temp = temps[blockIdx.x];
  const double hbar = 1.054571817e-34, kb = 1.380649e-23;
  double s = 0.0;
  if (temp > 0.0) {
    for (int i = threadIdx.x; i < W - 1; i += blockDim.x) {
      double f[2];
      for (int q = 0; q < 2; ++q) {
        const double wr = om[i + q] * unit;
        const double x = hbar * wr / (kb * temp);
        double ker = 0.0;
        if (x < 1e-6) ker = 1.0 - x * x / 12.0;
        else if (x < 700.0) {
          const double y = exp(-x);
          const double d = 1.0 - y;
          ker = x * x * y / (d * d);
        }
        f[q] = kb * tbar[i + q] * ker;
      }
      s += (om[i + 1] * unit - om[i] * unit) * (f[0] + f[1]) / 2.0;
    }
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[blockIdx.x] = (temp > 0.0) ? (1.0 / (2.0 * 3.141592653589793238462643383279502884)) * s : 0.0;
}

// Landauer heat current of each spectrum row b (block b):
//   J_b = (1/2pi) trapz((kB T_L phi(x_L) - kB T_R phi(x_R)) t_b(w), w),
//   phi(x) = x / expm1(x), x = hbar w / (kB T), with the series
//   1 - x/2 + x^2/12 below 1e-6 and 0 from 700 on (negfpy
//   core/thermal_current.py:30-67).
__device__ __forceinline__ double bose_phi(double x) {
  if (x < 1e-6) return 1.0 - 0.5 * x + (x * x) / 12.0;
  if (x < 700.0) return x / expm1(x);
  return 0.0;
}
__global__ void heat_current_kernel(const double* __restrict__ om, const double* __restrict__ t, int W, double temp_l,
                                    double temp_r, double* __restrict__ out) {
  __shared__ double red[40];
  const double hbar = 1.054571817e-34, kb = 1.380649e-23;
  const double* row = t + (long long)blockIdx.x * W;
  double s = 0.0;
  for (int i = threadIdx.x; i < W - 1; i += blockDim.x) {
    double f[2];
    for (int q = 0; q < 2; ++q) {
      const double w = om[i + q];
      // separately rounded products: equal temperatures cancel exactly
      const double wl = __dmul_rn(kb * temp_l, bose_phi(hbar * w / (kb * temp_l)));
      const double wr = __dmul_rn(kb * temp_r, bose_phi(hbar * w / (kb * temp_r)));
      f[q] = (wl - wr) * row[i + q];
    }
    s += (om[i + 1] - om[i]) * (f[0] + f[1]) / 2.0;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) out[blockIdx.x] = (1.0 / (2.0 * 3.141592653589793238462643383279502884)) * s;
}

// ---------------------------------------------------------------- launchers --
template <int NP>
static size_t smem_bytes() { return (size_t)6 * Geo<NP>::MAT * 16 + tail_bytes<NP>(); }
template <int NP>
static size_t sr_smem_bytes() {
  return (size_t)6 * Geo<NP>::MAT * 16 + tail_bytes<NP>() + (Split<NP>::on ? 4 * 32 * 16 : 0);  // + epsx
}

// Last launch failure of this host thread (read by the C-ABI layer).
thread_local char g_launch_err[256] = "";

template <typename K>
static int record_failure(const char* what, K kernel, cudaError_t e, size_t smem, int threads) {
  cudaFuncAttributes fa{};
  cudaFuncGetAttributes(&fa, kernel);
  snprintf(g_launch_err, sizeof(g_launch_err),
           "%s: %s (threads %d, dynamic smem %zu, regs %d, max threads %d, static smem %zu)", what,
           cudaGetErrorString(e), threads, smem, fa.numRegs, fa.maxThreadsPerBlock, fa.sharedSizeBytes);
  return -3;
}

const char* last_launch_error() { return g_launch_err; }

template <int NP>
static int launch_sr(const SrArgs& a, cudaStream_t st) {
  const size_t sm = sr_smem_bytes<NP>();
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(sr_f64_kernel<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return record_failure("sr_f64 smem attribute", sr_f64_kernel<NP>, e, sm, Geo<NP>::NTH);
    attr = true;
  }
  sr_f64_kernel<NP><<<a.batch, Geo<NP>::NTH, sm, st>>>(a);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : record_failure("sr_f64 launch", sr_f64_kernel<NP>, e, sm, Geo<NP>::NTH);
}

template <int NP>
static int launch_rgf(const RgfArgs& a, int grid, cudaStream_t st) {
  const size_t sm = smem_bytes<NP>();
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(rgf_f64_kernel<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return record_failure("rgf_f64 smem attribute", rgf_f64_kernel<NP>, e, sm, Geo<NP>::NTH);
    attr = true;
  }
  rgf_f64_kernel<NP><<<grid, Geo<NP>::NTH, sm, st>>>(a);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : record_failure("rgf_f64 launch", rgf_f64_kernel<NP>, e, sm, Geo<NP>::NTH);
}

template <int NP>
static int occupancy_rgf() {
  const size_t sm = smem_bytes<NP>();
  cudaFuncSetAttribute(rgf_f64_kernel<NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rgf_f64_kernel<NP>, Geo<NP>::NTH, sm) != cudaSuccess)
    return 0;
  return nb;
}

// Padded size for an order-n block: 1 (scalar path), 16, 32 or 48.
int padded_order(int n) {
  if (n == 1) return 1;
  if (n <= 16) return 16;
  if (n <= 32) return 32;
  if (n <= 48) return 48;
  return 0;
}

int sr_f64_launch(const SrArgs& a, cudaStream_t st) {
  if (a.batch <= 0) return 0;
  switch (padded_order(a.n)) {
    case 1: {
      const int tpb = 128;
      sr_scalar_kernel<<<(a.batch + tpb - 1) / tpb, tpb, 0, st>>>(a);
      return cudaGetLastError() == cudaSuccess ? 0 : -3;
    }
    case 16: return launch_sr<16>(a, st);
    case 32: return launch_sr<32>(a, st);
    case 48: return launch_sr<48>(a, st);
    default: return -2;
  }
}

int rgf_f64_grid(int np) {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  int per = 0;
  switch (np) {
    case 1: return 0;
    case 16: per = occupancy_rgf<16>(); break;
    case 32: per = occupancy_rgf<32>(); break;
    case 48: per = occupancy_rgf<48>(); break;
    default: return -2;
  }
  return per > 0 ? per * nsm : -3;
}

int rgf_f64_launch(const RgfArgs& a, int np, int grid, cudaStream_t st) {
  if (a.batch <= 0) return 0;
  switch (np) {
    case 1: {
      const int tpb = 128;
      rgf_scalar_kernel<<<(a.batch + tpb - 1) / tpb, tpb, 0, st>>>(a);
      return cudaGetLastError() == cudaSuccess ? 0 : -3;
    }
    case 16: return launch_rgf<16>(a, grid, st);
    case 32: return launch_rgf<32>(a, grid, st);
    case 48: return launch_rgf<48>(a, grid, st);
    default: return -2;
  }
}

int kavg_launch(const double* T, int W, int K, double* tbar, cudaStream_t st) {
  if (W <= 0) return 0;
  const int wpb = 8;
  kavg_kernel<<<(W + wpb - 1) / wpb, wpb * 32, 0, st>>>(T, W, K, tbar);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

int kmoments_launch(const double* T, int W, int K, double* t1, double* t2, cudaStream_t st) {
  if (W <= 0) return 0;
  const int wpb = 8;
  kmoments_kernel<<<(W + wpb - 1) / wpb, wpb * 32, 0, st>>>(T, W, K, t1, t2);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

int fcs_launch(const double* om, const double* t1, const double* t2, int W, double temp_l, double temp_r, double* out,
               cudaStream_t st) {
  fcs_kernel<<<1, 256, 0, st>>>(om, t1, t2, W, temp_l, temp_r, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

int heat_current_launch(const double* om, const double* t, int W, int n_spectra, double temp_l, double temp_r,
                        double* out, cudaStream_t st) {
  if (n_spectra <= 0) return 0;
  heat_current_kernel<<<n_spectra, 256, 0, st>>>(om, t, W, temp_l, temp_r, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

int kappa_launch(const double* om, const double* tbar, int W, const double* temps, int nT, double unit, double* out,
                 cudaStream_t st) {
  if (nT <= 0) return 0;
  kappa_kernel<<<nT, 256, 0, st>>>(om, tbar, W, temps, unit, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace negf
