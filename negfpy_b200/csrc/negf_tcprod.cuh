// Complex FP32 products on the fifth-generation tensor cores, for one thread
// block (kThreads = 256) working on one point's NP x NP matrices:
//
//   C = op(A) op(B),  op = identity or conjugate transpose,
//
// with A, B, C complex FP32 (interleaved re, im), row-major, row stride NP,
// NP a multiple of 16 and at most 128.  Each real product is split 3 x TF32
// (x = x_hi + x_lo, both TF32; x y ~ x_hi y_hi + x_hi y_lo + x_lo y_hi):
//
//   C_re = A_re B_re - A_im B_im,   C_im = A_re B_im + A_im B_re
//
// as twelve tcgen05.mma kind::tf32 (M = 128, N = NP, K = 8) per K step into
// two TMEM accumulators (C_re in columns [0, NP), C_im in [NP, 2 NP); rows
// >= NP of the M = 128 tile are zero), the A_im B_im terms with A negated in
// the instruction descriptor.  K runs in slabs of KS = 16: the block stages
// a slab of both operands in shared memory (split and laid out in the
// no-swizzle K-major core-matrix layout), one thread issues the slab's 24
// MMAs and commits them to an mbarrier while every thread loads the next
// slab from global memory into registers, every thread waits on the barrier
// (at most 2 s of wall time; then the product reports failure), and the next
// slab is staged.  The result is read back with tcgen05.ld and
// written to C.
#pragma once
#include "negf_common.cuh"
#include "negf_tiles.cuh"
#include "negf_umma.cuh"

namespace negf {
namespace tc {

using glob::kThreads;
constexpr int KS = 16;               // K per staged slab: two MMA steps of 8
constexpr int MT = 128;              // MMA tile rows (M)
constexpr int kMaxNP = 128;
constexpr int kTmemCols = 256;       // 2 kMaxNP FP32 columns
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s per slab: far above any real completion time

// Shared memory of the product: 4 A parts (128 x KS) and 4 B parts (NP x KS).
__host__ __device__ constexpr size_t stage_bytes(int np) { return (size_t)4 * MT * KS * 4 + (size_t)4 * np * KS * 4; }

struct Ctx {
  float* stage;     // shared, stage_bytes(NP), 128-byte aligned
  uint64_t* bar;    // shared mbarrier, initialised with count 1
  uint32_t tmem;    // TMEM base address, kTmemCols columns
  uint32_t phase;   // parity of the next mbarrier phase (same in every thread)
  int* err;         // shared flag, set when a wait runs out
};

// Byte offset of element (r, k) in a part of the slab (8-row x 16-byte core
// matrices; KS / 4 core matrices per 8-row group).
__device__ __forceinline__ uint32_t core_off(int r, int k) {
  return (uint32_t)(((r >> 3) * (KS / 4) + (k >> 2)) * 128 + (r & 7) * 16 + (k & 3) * 4);
}
__device__ __forceinline__ void put_split(unsigned char* part0, uint32_t part_bytes, uint32_t off, float2 v) {
  unsigned rh, rl, ih, il;
  split_tf32(v.x, rh, rl);
  split_tf32(v.y, ih, il);
  *reinterpret_cast<unsigned*>(part0 + off) = rh;
  *reinterpret_cast<unsigned*>(part0 + part_bytes + off) = rl;
  *reinterpret_cast<unsigned*>(part0 + 2 * part_bytes + off) = ih;
  *reinterpret_cast<unsigned*>(part0 + 3 * part_bytes + off) = il;
}

// Elements of one slab a thread stages: MT*KS of A and NP*KS of B over the
// block's threads (at most kMaxNP).
constexpr int kPerA = MT * KS / kThreads;
constexpr int kPerB = kMaxNP * KS / kThreads;

template <bool AC>
__device__ __forceinline__ void load_a(float2 (&ra)[kPerA], const float2* __restrict__ A, int NP, int k0) {
#pragma unroll
  for (int i = 0; i < kPerA; ++i) {
    const int e = threadIdx.x + i * kThreads;
    int r, k;
    if (AC) { k = e / MT; r = e - k * MT; } else { r = e / KS; k = e - r * KS; }
    float2 v = make_float2(0.f, 0.f);
    if (r < NP) {
      v = AC ? A[(long long)(k0 + k) * NP + r] : A[(long long)r * NP + k0 + k];
      if (AC) v.y = -v.y;
    }
    ra[i] = v;
  }
}
template <bool BC>
__device__ __forceinline__ void load_b(float2 (&rb)[kPerB], const float2* __restrict__ B, int NP, int k0) {
#pragma unroll
  for (int i = 0; i < kPerB; ++i) {
    const int e = threadIdx.x + i * kThreads;
    float2 v = make_float2(0.f, 0.f);
    if (e < NP * KS) {
      int n, k;
      if (BC) { n = e / KS; k = e - n * KS; } else { k = e / NP; n = e - k * NP; }
      v = BC ? B[(long long)n * NP + k0 + k] : B[(long long)(k0 + k) * NP + n];
      if (BC) v.y = -v.y;
    }
    rb[i] = v;
  }
}

// C = op(A) op(B).  Every thread of the block calls it; it ends with the
// block synchronised.  Returns false if an mbarrier wait ran out (C is then
// not valid; *ctx.err is set).  The global loads of slab s + 1 are issued
// right after slab s's MMAs, so they overlap the MMAs and the wait.
template <bool AC, bool BC>
__device__ bool cprod(float2* __restrict__ C, const float2* __restrict__ A, const float2* __restrict__ B, int NP,
                      Ctx& ctx) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  unsigned char* sa = reinterpret_cast<unsigned char*>(ctx.stage);
  const uint32_t pa_bytes = MT * KS * 4;
  unsigned char* sb = sa + 4 * pa_bytes;
  const uint32_t pb_bytes = (uint32_t)NP * KS * 4;
  const uint32_t lbo = 128, sbo = (KS / 4) * 128;
  const uint32_t id_pos = umma::idesc_tf32(MT, NP, false), id_neg = umma::idesc_tf32(MT, NP, true);
  const uint32_t t_re = ctx.tmem, t_im = ctx.tmem + (uint32_t)NP;
  bool ok = true;
  float2 ra[kPerA], rb[kPerB];
  load_a<AC>(ra, A, NP, 0);
  load_b<BC>(rb, B, NP, 0);
  for (int k0 = 0; k0 < NP; k0 += KS) {
    // stage op(A)[0:128, k0:k0+KS] and op(B)[k0:k0+KS, 0:NP] (as its transpose)
#pragma unroll
    for (int i = 0; i < kPerA; ++i) {
      const int e = tid + i * kThreads;
      int r, k;
      if (AC) { k = e / MT; r = e - k * MT; } else { r = e / KS; k = e - r * KS; }
      put_split(sa, pa_bytes, core_off(r, k), ra[i]);
    }
#pragma unroll
    for (int i = 0; i < kPerB; ++i) {
      const int e = tid + i * kThreads;
      if (e < NP * KS) {
        int n, k;
        if (BC) { n = e / KS; k = e - n * KS; } else { k = e / NP; n = e - k * NP; }
        put_split(sb, pb_bytes, core_off(n, k), rb[i]);
      }
    }
    umma::fence_proxy_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (tid == 0 && ok) {
      for (int s = 0; s < KS / 8; ++s) {
        const bool first = (k0 == 0 && s == 0);
        uint64_t ad[4], bd[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          ad[q] = umma::smem_desc(sa + q * pa_bytes + s * 256, lbo, sbo);
          bd[q] = umma::smem_desc(sb + q * pb_bytes + s * 256, lbo, sbo);
        }
        // parts: 0 re_hi, 1 re_lo, 2 im_hi, 3 im_lo; small terms first
        umma::mma_tf32(t_re, ad[1], bd[0], id_pos, !first);
        umma::mma_tf32(t_re, ad[0], bd[1], id_pos, true);
        umma::mma_tf32(t_re, ad[3], bd[2], id_neg, true);
        umma::mma_tf32(t_re, ad[2], bd[3], id_neg, true);
        umma::mma_tf32(t_re, ad[0], bd[0], id_pos, true);
        umma::mma_tf32(t_re, ad[2], bd[2], id_neg, true);
        umma::mma_tf32(t_im, ad[1], bd[2], id_pos, !first);
        umma::mma_tf32(t_im, ad[0], bd[3], id_pos, true);
        umma::mma_tf32(t_im, ad[3], bd[0], id_pos, true);
        umma::mma_tf32(t_im, ad[2], bd[1], id_pos, true);
        umma::mma_tf32(t_im, ad[0], bd[2], id_pos, true);
        umma::mma_tf32(t_im, ad[2], bd[0], id_pos, true);
      }
      umma::mma_commit(ctx.bar);
    }
    if (k0 + KS < NP) {  // next slab's operands, in flight during the MMAs
      load_a<AC>(ra, A, NP, k0 + KS);
      load_b<BC>(rb, B, NP, k0 + KS);
    }
    if (ok) {
      ok = umma::mbar_wait(ctx.bar, ctx.phase, kWaitLimitNs);
      ctx.phase ^= 1u;
    }
    if (!ok && lane == 0) *ctx.err = 1;
    ok = __syncthreads_and(ok);  // also: the slab may be overwritten now
    umma::fence_after_sync();
  }
  if (ok) {
    // read back: warp w takes rows 32 (w % 4) + lane and half (w / 4) of the columns
    const int lb = 32 * (warp & 3), half = NP / 2, c0 = (warp >> 2) * half;
    const int r = lb + lane;
    const uint32_t lane_base = (uint32_t)lb << 16;
    for (int c = c0; c < c0 + half; c += 8) {
      float re[8], im[8];
      umma::tmem_ld8(t_re + lane_base + (uint32_t)c, re);
      umma::tmem_ld8(t_im + lane_base + (uint32_t)c, im);
      if (r < NP) {
#pragma unroll
        for (int i = 0; i < 8; ++i) C[(long long)r * NP + c + i] = make_float2(re[i], im[i]);
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  return ok;
}

// Shared-memory set-up for a block that uses cprod: carve the stage and the
// mbarrier, allocate TMEM (warp 0), initialise the barrier.  `raw` must be
// 128-byte aligned with stage_bytes(NP) + 16 bytes; `tslot` a shared word.
__device__ __forceinline__ Ctx setup(unsigned char* raw, int NP, uint32_t* tslot, int* err) {
  Ctx c;
  c.stage = reinterpret_cast<float*>(raw);
  c.bar = reinterpret_cast<uint64_t*>(raw + stage_bytes(NP));
  c.err = err;
  if ((threadIdx.x >> 5) == 0) umma::tmem_alloc(tslot, kTmemCols);
  if (threadIdx.x == 0) {
    umma::mbar_init(c.bar, 1);
    *err = 0;
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  c.tmem = *tslot;
  c.phase = 0;
  return c;
}
__device__ __forceinline__ void teardown(const Ctx& c) {
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if ((threadIdx.x >> 5) == 0) umma::tmem_dealloc(c.tmem, kTmemCols);
}

}  // namespace tc
}  // namespace negf
