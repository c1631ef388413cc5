// FP64 kernels of the per-(omega, k) phonon NEGF path.
//
// One thread block owns one (omega, k) point at a time.  Blocks of order
// n <= 48 live entirely in shared memory, padded to NP (a multiple of the
// thread-grid side TG) with a row stride of NP + 1 complex numbers so that
// row and column walks are both bank-conflict free.  Thread (tr, tc) of the
// TG x TG grid owns the RT x RT elements (tr + TG*i, tc + TG*j), RT = NP/TG,
// in every matrix operation (products, Gauss-Jordan updates, epilogues), so
// register-resident matrices line up with shared-memory ones.
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
#include "negf_common.cuh"
#include "negf_f64.h"

namespace negf {

// z = (omega + i eta)^2 with the two products rounded separately, as the
// reference's complex power does (no fused multiply-add in the real part).
__device__ __forceinline__ double2 z_of(double w, double e) {
  return make_double2(__dsub_rn(__dmul_rn(w, w), __dmul_rn(e, e)), __dmul_rn(2.0 * w, e));
}

template <int NP, int TG>
struct Geo {
  static constexpr int RT = NP / TG;
  static constexpr int LD = NP + 1;
  static constexpr int MAT = NP * LD;  // complex elements per matrix buffer
  static constexpr int NTH = TG * TG;
};

// ---------------------------------------------------------------- products --
// c = op(A) op(B) summed over k < kn; op = conjugate transpose when AC / BC.
template <int NP, int TG, bool AC, bool BC>
__device__ __forceinline__ void mm(double2 (&c)[NP / TG][NP / TG], const double2* __restrict__ A,
                                   const double2* __restrict__ B, int kn, int tr, int tc) {
  constexpr int RT = NP / TG, LD = NP + 1;
#pragma unroll
  for (int i = 0; i < RT; ++i)
#pragma unroll
    for (int j = 0; j < RT; ++j) c[i][j] = make_double2(0.0, 0.0);
#pragma unroll 2
  for (int k = 0; k < kn; ++k) {
    double2 a[RT], b[RT];
#pragma unroll
    for (int i = 0; i < RT; ++i) a[i] = AC ? cconj(A[k * LD + tr + TG * i]) : A[(tr + TG * i) * LD + k];
#pragma unroll
    for (int j = 0; j < RT; ++j) b[j] = BC ? cconj(B[(tc + TG * j) * LD + k]) : B[k * LD + tc + TG * j];
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int j = 0; j < RT; ++j) cfma(c[i][j], a[i], b[j]);
  }
}

// c1 = A1 B, c2 = A2 B: two products sharing the right operand.
template <int NP, int TG>
__device__ __forceinline__ void mm2b(double2 (&c1)[NP / TG][NP / TG], double2 (&c2)[NP / TG][NP / TG],
                                     const double2* __restrict__ A1, const double2* __restrict__ A2,
                                     const double2* __restrict__ B, int kn, int tr, int tc) {
  constexpr int RT = NP / TG, LD = NP + 1;
#pragma unroll
  for (int i = 0; i < RT; ++i)
#pragma unroll
    for (int j = 0; j < RT; ++j) c1[i][j] = c2[i][j] = make_double2(0.0, 0.0);
#pragma unroll 2
  for (int k = 0; k < kn; ++k) {
    double2 a1[RT], a2[RT], b[RT];
#pragma unroll
    for (int j = 0; j < RT; ++j) b[j] = B[k * LD + tc + TG * j];
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      a1[i] = A1[(tr + TG * i) * LD + k];
      a2[i] = A2[(tr + TG * i) * LD + k];
    }
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        cfma(c1[i][j], a1[i], b[j]);
        cfma(c2[i][j], a2[i], b[j]);
      }
  }
}

// c1 = A1 B1, c2 = A2 B2.
template <int NP, int TG>
__device__ __forceinline__ void mmpair(double2 (&c1)[NP / TG][NP / TG], double2 (&c2)[NP / TG][NP / TG],
                                       const double2* __restrict__ A1, const double2* __restrict__ B1,
                                       const double2* __restrict__ A2, const double2* __restrict__ B2, int kn,
                                       int tr, int tc) {
  constexpr int RT = NP / TG, LD = NP + 1;
#pragma unroll
  for (int i = 0; i < RT; ++i)
#pragma unroll
    for (int j = 0; j < RT; ++j) c1[i][j] = c2[i][j] = make_double2(0.0, 0.0);
#pragma unroll 2
  for (int k = 0; k < kn; ++k) {
    double2 a1[RT], a2[RT], b1[RT], b2[RT];
#pragma unroll
    for (int j = 0; j < RT; ++j) {
      b1[j] = B1[k * LD + tc + TG * j];
      b2[j] = B2[k * LD + tc + TG * j];
    }
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      a1[i] = A1[(tr + TG * i) * LD + k];
      a2[i] = A2[(tr + TG * i) * LD + k];
    }
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        cfma(c1[i][j], a1[i], b1[j]);
        cfma(c2[i][j], a2[i], b2[j]);
      }
  }
}

template <int NP, int TG>
__device__ __forceinline__ void store_tile(double2* S, const double2 (&c)[NP / TG][NP / TG], int tr, int tc) {
  constexpr int RT = NP / TG, LD = NP + 1;
#pragma unroll
  for (int i = 0; i < RT; ++i)
#pragma unroll
    for (int j = 0; j < RT; ++j) S[(tr + TG * i) * LD + tc + TG * j] = c[i][j];
}

// Global n_r x n_c row-major matrix -> padded shared buffer (zeros outside).
template <int NP, int TG>
__device__ __forceinline__ void load_mat(double2* S, const double2* __restrict__ G, int nr, int nc) {
  constexpr int LD = NP + 1, NTH = TG * TG;
  for (int idx = threadIdx.x; idx < NP * NP; idx += NTH) {
    int r = idx / NP, c = idx - r * NP;
    S[r * LD + c] = (r < nr && c < nc) ? G[(long long)r * nc + c] : make_double2(0.0, 0.0);
  }
}

// ---------------------------------------------------------- Gauss-Jordan --
// In-place inverse of the leading n x n block of M (the padding must hold the
// identity) by Gauss-Jordan elimination with partial pivoting on |re| + |im|
// (the pivot measure of LAPACK's getrf).  Row interchanges are undone as
// column interchanges at the end.  Returns kOk, kSingular (exact zero pivot)
// or kNonFinite, identically in every thread.
struct GJScratch {
  double2* rowk;   // scaled pivot row
  double2* colk;   // pivot column after the interchange
  double2* oldrk;  // pivot row before the interchange
  int* perm;       // interchange record
  int* piv;        // [0] pivot row, [1] status
};

template <int NP, int TG>
__device__ int gj_invert(double2* M, int n, const GJScratch& s) {
  constexpr int RT = NP / TG, LD = NP + 1, NTH = TG * TG;
  const int tid = threadIdx.x, tr = tid / TG, tc = tid - tr * TG;
  for (int k = 0; k < n; ++k) {
    if (tid < 32) {
      double best = -1.0;
      int bi = n;
      for (int i = k + tid; i < n; i += 32) {
        double v = cabs1(M[i * LD + k]);
        if (v > best) { best = v; bi = i; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
      }
      if (tid == 0) {
        s.piv[0] = bi;
        s.piv[1] = (best > 0.0) ? (int)kOk : (best == 0.0 ? (int)kSingular : (int)kNonFinite);
      }
    }
    __syncthreads();
    const int pr = s.piv[0];
    const int bad = s.piv[1];
    if (bad) return bad;
    const double2 piv = M[pr * LD + k];
    const double2 ip = crecip(piv);
    for (int t = tid; t < n; t += NTH) {
      double2 rk = M[k * LD + t];
      s.oldrk[t] = rk;
      s.rowk[t] = (t == k) ? ip : cmul(M[pr * LD + t], ip);
      s.colk[t] = (t == k) ? piv : ((t == pr) ? M[k * LD + k] : M[t * LD + k]);
    }
    if (tid == 0) s.perm[k] = pr;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RT; ++i) {
      const int r = tr + TG * i;
      if (r >= n) continue;
      const double2 ci = s.colk[r];
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        const int c = tc + TG * j;
        if (c >= n) continue;
        double2 v;
        if (r == k) {
          v = s.rowk[c];
        } else if (c == k) {
          v = cneg(cmul(ci, ip));
        } else {
          v = (r == pr) ? s.oldrk[c] : M[r * LD + c];
          cfma(v, cneg(ci), s.rowk[c]);
        }
        M[r * LD + c] = v;
      }
    }
    __syncthreads();
  }
  for (int r = tid; r < n; r += NTH) {
    for (int k = n - 1; k >= 0; --k) {
      const int q = s.perm[k];
      if (q != k) {
        double2 t = M[r * LD + k];
        M[r * LD + k] = M[r * LD + q];
        M[r * LD + q] = t;
      }
    }
  }
  __syncthreads();
  return kOk;
}

template <int NP, int TG>
__device__ __forceinline__ GJScratch carve_gj(double2* base) {
  GJScratch s;
  s.rowk = base;
  s.colk = base + NP;
  s.oldrk = base + 2 * NP;
  s.perm = reinterpret_cast<int*>(base + 3 * NP);
  s.piv = s.perm + NP;
  return s;
}
// Bytes after the matrix buffers: GJ vectors, perm/pivot ints, reduction slots.
template <int NP>
constexpr int tail_bytes() { return 3 * NP * 16 + ((NP + 4) * 4 + 15) / 16 * 16 + 40 * 8; }

// ------------------------------------------------------------ Sancho-Rubio --
template <int NP, int TG>
__global__ void __launch_bounds__(TG* TG, 1) sr_f64_kernel(SrArgs a) {
  using G = Geo<NP, TG>;
  constexpr int RT = G::RT, LD = G::LD, MAT = G::MAT;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* sA = reinterpret_cast<double2*>(smraw);
  double2* sB = sA + MAT;
  double2* sG = sB + MAT;
  double2* sAG = sG + MAT;
  double2* sBG = sAG + MAT;
  double2* tail = sBG + MAT;
  GJScratch gs = carve_gj<NP, TG>(tail);
  double* red = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(tail) + 3 * NP * 16 +
                                          ((NP + 4) * 4 + 15) / 16 * 16);

  const int p = blockIdx.x;
  if (p >= a.batch) return;
  const int n = a.n;
  const int tid = threadIdx.x, tr = tid / TG, tc = tid - tr * TG;
  const long long kset = a.kidx ? (long long)a.kidx[p] : 0;
  const double2* h00 = a.h00 + kset * a.lead_stride;
  const double2* h01 = a.h01 + kset * a.lead_stride;
  const double2* h10 = a.h10 ? a.h10 + kset * a.lead_stride : nullptr;
  const double w = a.omega[p];
  const double2 z = z_of(w, a.eta[p]);

  double2 eps[RT][RT], epss[RT][RT];
#pragma unroll
  for (int i = 0; i < RT; ++i)
#pragma unroll
    for (int j = 0; j < RT; ++j) {
      const int r = tr + TG * i, c = tc + TG * j;
      double2 e = (r < n && c < n) ? h00[r * n + c] : make_double2(0.0, 0.0);
      eps[i][j] = e;
      epss[i][j] = e;
    }
  for (int idx = tid; idx < NP * NP; idx += G::NTH) {
    const int r = idx / NP, c = idx - r * NP;
    const bool in = r < n && c < n;
    sA[r * LD + c] = in ? h01[r * n + c] : make_double2(0.0, 0.0);
    sB[r * LD + c] = in ? (h10 ? h10[r * n + c] : cconj(h01[c * n + r])) : make_double2(0.0, 0.0);
  }

  int status = kOk;
  int it = 0;
  const double tol2 = a.tol * a.tol;
  double2 c1[RT][RT], c2[RT][RT];
  bool converged = false;
  for (it = 1; it <= a.maxiter; ++it) {
    // M = z - eps (identity in the padding), inverted in place.
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        const int r = tr + TG * i, c = tc + TG * j;
        double2 v;
        if (r < n && c < n) v = (r == c) ? csub(z, eps[i][j]) : cneg(eps[i][j]);
        else v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        sG[r * LD + c] = v;
      }
    __syncthreads();
    status = gj_invert<NP, TG>(sG, n, gs);
    if (status != kOk) break;
    // alpha g, beta g
    mm2b<NP, TG>(c1, c2, sA, sB, sG, n, tr, tc);
    store_tile<NP, TG>(sAG, c1, tr, tc);
    store_tile<NP, TG>(sBG, c2, tr, tc);
    __syncthreads();
    // eps_s += (alpha g) beta ; eps += (alpha g) beta + (beta g) alpha
    mmpair<NP, TG>(c1, c2, sAG, sB, sBG, sA, n, tr, tc);
    int bad = 0;
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        epss[i][j] = cadd(epss[i][j], c1[i][j]);
        eps[i][j] = cadd(cadd(eps[i][j], c1[i][j]), c2[i][j]);
        bad |= !cfinite(epss[i][j]) || !cfinite(eps[i][j]);
      }
    // alpha <- (alpha g) alpha ; beta <- (beta g) beta
    mmpair<NP, TG>(c1, c2, sAG, sA, sBG, sB, n, tr, tc);
    double e2 = 0.0;
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        bad |= !cfinite(c1[i][j]) || !cfinite(c2[i][j]);
        e2 = fmax(e2, fmax(cabs2(c1[i][j]), cabs2(c2[i][j])));
      }
    __syncthreads();  // every read of alpha and beta is done
    store_tile<NP, TG>(sA, c1, tr, tc);
    store_tile<NP, TG>(sB, c2, tr, tc);
    if (block_any(bad)) { status = kNonFinite; break; }
    const double emax = block_max(e2, red);
    if (emax < tol2) { converged = true; break; }
  }
  if (status == kOk && !converged) {
    status = kMaxIter;
    it = a.maxiter;
  }
  if (status == kOk) {
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        const int r = tr + TG * i, c = tc + TG * j;
        double2 v;
        if (r < n && c < n) v = (r == c) ? csub(z, epss[i][j]) : cneg(epss[i][j]);
        else v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        sG[r * LD + c] = v;
      }
    __syncthreads();
    status = gj_invert<NP, TG>(sG, n, gs);
  }
  if (status == kOk) {
    if (a.g_out) {
      double2* go = a.g_out + (long long)p * n * n;
      for (int idx = tid; idx < n * n; idx += G::NTH) {
        const int r = idx / n, c = idx - r * n;
        go[idx] = sG[r * LD + c];
      }
    }
    if (a.dos_out) {
      // (omega/pi) Re Tr[i (g - g^H)] = (omega/pi) sum_j (-2 Im g_jj)
      double t = 0.0;
      for (int j = tid; j < n; j += G::NTH) t += -2.0 * sG[j * LD + j].y;
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
template <int NP, int TG>
__global__ void __launch_bounds__(TG* TG, 1) rgf_f64_kernel(RgfArgs a) {
  using G = Geo<NP, TG>;
  constexpr int RT = G::RT, LD = G::LD, MAT = G::MAT;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* bG = reinterpret_cast<double2*>(smraw);  // left-connected g_i
  double2* bC = bG + MAT;                             // coupling C_{i-1}
  double2* bW = bC + MAT;                             // g_{i-1} C_{i-1}
  double2* bU = bW + MAT;                             // G_{0,i-1} C_{i-1}
  double2* bG0 = bU + MAT;                            // G_{0,i}
  double2* tail = bG0 + MAT;
  GJScratch gs = carve_gj<NP, TG>(tail);
  double* red = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(tail) + 3 * NP * 16 +
                                          ((NP + 4) * 4 + 15) / 16 * 16);
  __shared__ int s_point;

  const int n = a.n, L = a.L;
  const int tid = threadIdx.x, tr = tid / TG, tc = tid - tr * TG;
  double2* sigL = a.sigma_ws + (long long)blockIdx.x * 2 * n * n;
  double2* sigR = sigL + (long long)n * n;
  double2 c1[RT][RT], c2[RT][RT];

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

    // Contact self-energies Sigma = V g V^H into this block's scratch.
    for (int side = 0; side < 2; ++side) {
      const int nl = side ? a.nr : a.nl;
      const double2* V = side ? a.VR + k * a.vr_ks : a.VL + k * a.vl_ks;
      const double2* g = side ? a.gR + (long long)p * a.gr_ps : a.gL + (long long)p * a.gl_ps;
      double2* S = side ? sigR : sigL;
      load_mat<NP, TG>(bC, V, n, nl);
      load_mat<NP, TG>(bW, g, nl, nl);
      __syncthreads();
      mm<NP, TG, false, false>(c1, bC, bW, nl, tr, tc);
      store_tile<NP, TG>(bU, c1, tr, tc);
      __syncthreads();
      mm<NP, TG, false, true>(c1, bU, bC, nl, tr, tc);
#pragma unroll
      for (int i = 0; i < RT; ++i)
#pragma unroll
        for (int j = 0; j < RT; ++j) {
          const int r = tr + TG * i, c = tc + TG * j;
          if (r < n && c < n) S[r * n + c] = c1[i][j];
        }
      __syncthreads();
    }

    // Layer 0: g_0 = (z - D_0 - Sigma_L [- Sigma_R when L == 1])^-1 = G_{0,0}.
#pragma unroll
    for (int i = 0; i < RT; ++i)
#pragma unroll
      for (int j = 0; j < RT; ++j) {
        const int r = tr + TG * i, c = tc + TG * j;
        double2 v;
        if (r < n && c < n) {
          v = csub(cneg(D[r * n + c]), sigL[r * n + c]);
          if (L == 1) v = csub(v, sigR[r * n + c]);
          if (r == c) v = cadd(v, z);
        } else {
          v = make_double2(r == c ? 1.0 : 0.0, 0.0);
        }
        bG[r * LD + c] = v;
      }
    __syncthreads();
    int status = gj_invert<NP, TG>(bG, n, gs);
    if (status == kOk) {
#pragma unroll
      for (int i = 0; i < RT; ++i)
#pragma unroll
        for (int j = 0; j < RT; ++j) {
          const int r = tr + TG * i, c = tc + TG * j;
          bG0[r * LD + c] = bG[r * LD + c];
        }
      for (int l = 1; l < L && status == kOk; ++l) {
        load_mat<NP, TG>(bC, C + (long long)(l - 1) * a.c_ls, n, n);
        __syncthreads();
        // W = g_{l-1} C, U = G_{0,l-1} C
        mm2b<NP, TG>(c1, c2, bG, bG0, bC, n, tr, tc);
        store_tile<NP, TG>(bW, c1, tr, tc);
        store_tile<NP, TG>(bU, c2, tr, tc);
        __syncthreads();
        // M = z - D_l - C^H W [- Sigma_R on the last layer]
        mm<NP, TG, true, false>(c1, bC, bW, n, tr, tc);
        const double2* Dl = D + (long long)l * a.d_ls;
        const bool last = (l == L - 1);
#pragma unroll
        for (int i = 0; i < RT; ++i)
#pragma unroll
          for (int j = 0; j < RT; ++j) {
            const int r = tr + TG * i, c = tc + TG * j;
            double2 v;
            if (r < n && c < n) {
              v = csub(cneg(Dl[r * n + c]), c1[i][j]);
              if (last) v = csub(v, sigR[r * n + c]);
              if (r == c) v = cadd(v, z);
            } else {
              v = make_double2(r == c ? 1.0 : 0.0, 0.0);
            }
            bG[r * LD + c] = v;
          }
        __syncthreads();
        status = gj_invert<NP, TG>(bG, n, gs);
        if (status != kOk) break;
        // G_{0,l} = U g_l
        mm<NP, TG, false, false>(c1, bU, bG, n, tr, tc);
        store_tile<NP, TG>(bG0, c1, tr, tc);
        __syncthreads();
      }
    }
    double tval = 0.0;
    if (status == kOk) {
      // Gamma = i (Sigma - Sigma^H) for both contacts.
#pragma unroll
      for (int i = 0; i < RT; ++i)
#pragma unroll
        for (int j = 0; j < RT; ++j) {
          const int r = tr + TG * i, c = tc + TG * j;
          double2 gl = make_double2(0.0, 0.0), gr = gl;
          if (r < n && c < n) {
            double2 d = csub(sigL[r * n + c], cconj(sigL[c * n + r]));
            gl = make_double2(-d.y, d.x);
            d = csub(sigR[r * n + c], cconj(sigR[c * n + r]));
            gr = make_double2(-d.y, d.x);
          }
          bC[r * LD + c] = gl;
          bW[r * LD + c] = gr;
        }
      __syncthreads();
      mm<NP, TG, false, false>(c1, bC, bG0, n, tr, tc);
      store_tile<NP, TG>(bU, c1, tr, tc);
      __syncthreads();
      mm<NP, TG, false, false>(c1, bU, bW, n, tr, tc);
      double t = 0.0;
#pragma unroll
      for (int i = 0; i < RT; ++i)
#pragma unroll
        for (int j = 0; j < RT; ++j) {
          const int r = tr + TG * i, c = tc + TG * j;
          const double2 g = bG0[r * LD + c];
          t += c1[i][j].x * g.x + c1[i][j].y * g.y;
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
    if (!cfinite(es) || !cfinite(e) || !cfinite(al) || !cfinite(be)) { status = kNonFinite; break; }
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

// ---------------------------------------------------------------- launchers --
template <int NP, int TG>
static size_t smem_bytes() { return (size_t)5 * Geo<NP, TG>::MAT * 16 + tail_bytes<NP>(); }

template <int NP, int TG>
static int launch_sr(const SrArgs& a, cudaStream_t st) {
  const size_t sm = smem_bytes<NP, TG>();
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(sr_f64_kernel<NP, TG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
      return -3;
    attr = true;
  }
  sr_f64_kernel<NP, TG><<<a.batch, TG * TG, sm, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

template <int NP, int TG>
static int launch_rgf(const RgfArgs& a, int grid, cudaStream_t st) {
  const size_t sm = smem_bytes<NP, TG>();
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(rgf_f64_kernel<NP, TG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
      return -3;
    attr = true;
  }
  rgf_f64_kernel<NP, TG><<<grid, TG * TG, sm, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

template <int NP, int TG>
static int occupancy_rgf() {
  const size_t sm = smem_bytes<NP, TG>();
  cudaFuncSetAttribute(rgf_f64_kernel<NP, TG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, rgf_f64_kernel<NP, TG>, TG * TG, sm) != cudaSuccess) return 0;
  return nb;
}

// Padded size for an order-n block: 1 (scalar path), 8, 16, 24, 32 or 48.
int padded_order(int n) {
  if (n == 1) return 1;
  if (n <= 8) return 8;
  if (n <= 16) return 16;
  if (n <= 24) return 24;
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
    case 8: return launch_sr<8, 8>(a, st);
    case 16: return launch_sr<16, 8>(a, st);
    case 24: return launch_sr<24, 8>(a, st);
    case 32: return launch_sr<32, 16>(a, st);
    case 48: return launch_sr<48, 16>(a, st);
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
    case 8: per = occupancy_rgf<8, 8>(); break;
    case 16: per = occupancy_rgf<16, 8>(); break;
    case 24: per = occupancy_rgf<24, 8>(); break;
    case 32: per = occupancy_rgf<32, 16>(); break;
    case 48: per = occupancy_rgf<48, 16>(); break;
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
    case 8: return launch_rgf<8, 8>(a, grid, st);
    case 16: return launch_rgf<16, 8>(a, grid, st);
    case 24: return launch_rgf<24, 8>(a, grid, st);
    case 32: return launch_rgf<32, 16>(a, grid, st);
    case 48: return launch_rgf<48, 16>(a, grid, st);
    default: return -2;
  }
}

int kavg_launch(const double* T, int W, int K, double* tbar, cudaStream_t st) {
  if (W <= 0) return 0;
  const int wpb = 8;
  kavg_kernel<<<(W + wpb - 1) / wpb, wpb * 32, 0, st>>>(T, W, K, tbar);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

int kappa_launch(const double* om, const double* tbar, int W, const double* temps, int nT, double unit, double* out,
                 cudaStream_t st) {
  if (nT <= 0) return 0;
  kappa_kernel<<<nT, 256, 0, st>>>(om, tbar, W, temps, unit, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace negf
