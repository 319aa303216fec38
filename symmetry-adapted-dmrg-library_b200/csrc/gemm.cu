// gemm.cu -- grouped block-GEMM executor with deterministic split-K.
//
// A plan is a list of jobs (output blocks C, m x n) with accumulation lists of
// terms alpha * op(A) * op(B).  Work is cut into items of one output tile and a
// contiguous range of the job's concatenated reduction dimension (the k of all
// its terms laid end to end), so a matvec with a few large output blocks still
// fills all 148 SMs.  An item that covers the whole range writes C directly;
// otherwise it writes its partial tile to a workspace slot, and the last item of
// the tile to finish sums the slots in a fixed order -- results are bitwise
// reproducible and there is no separate reduction launch.
//
// Inner loop: operand slabs (BM x BK and BK x BN) are prefetched into registers
// while the tensor cores work on the slab already in shared memory (two shared
// buffers, one barrier per slab).  Transposes, conjugation and the term's alpha
// are applied on the register -> shared store.
//   FP64   : mma.sync m8n8k4 .f64 (the double-precision tensor path; tcgen05 has
//            no f64 kind), 64 x 64 tiles, 4 warps of 32 x 32.
//   3xTF32 : x = hi + lo with hi = tf32(x), lo = tf32(x - hi); hi*hi + hi*lo +
//            lo*hi on mma.sync m16n8k8 .tf32 with FP32 partial sums folded into
//            FP64 registers after every slab (Markidis et al. 2018; Ootomo &
//            Yokota 2022).
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include <type_traits>

#include "kernels.cuh"

namespace sadmrg {

constexpr int kThreads = 128;

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split3(double v, uint32_t& hi, uint32_t& lo) {
  const float f = (float)v;
  hi = to_tf32(f);
  lo = to_tf32(f - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Walk over the slabs of an item: term index t (absolute), offset k inside the term,
// slab width kt (< BK at a term end or at the end of the item's range).
struct SlabWalk {
  int t, k, rem;
  __device__ bool next(const GemmTerm* terms, int BK, int& tt, int& kk, int& kt) {
    if (rem <= 0) return false;
    int tk = terms[t].k;
    while (k >= tk) { ++t; k = 0; tk = terms[t].k; }
    tt = t;
    kk = k;
    kt = min(BK, min(tk - k, rem));
    k += kt;
    rem -= kt;
    return true;
  }
};

// per-thread register slab: A is BM x BK, B is BK x BN (after op), E = elements per thread
template <class V, int BM, int BN, int BK>
struct Slab {
  static constexpr int EA = BM * BK / kThreads, EB = BK * BN / kThreads;
  V a[EA], b[EB];

  __device__ __forceinline__ void load(const GemmTerm& T, const GemmJob& J, int row0, int col0, int k0, int kt,
                                       const Bases& bases) {
    const V* A = static_cast<const V*>(bases.p[T.abuf]) + T.aoff;
    const V* B = static_cast<const V*>(bases.p[T.bbuf]) + T.boff;
    const bool ta = T.flags & TF_TA, tb = T.flags & TF_TB;
    const int tid = threadIdx.x;
#pragma unroll
    for (int q = 0; q < EA; ++q) {
      const int e = tid + q * kThreads;
      int i, kk;
      if (!ta) { i = e % BM; kk = e / BM; } else { kk = e % BK; i = e / BK; }
      const int gi = row0 + i;
      V v = zero();
      if (gi < J.m && kk < kt) v = ta ? A[(k0 + kk) + (long long)gi * T.lda] : A[gi + (long long)(k0 + kk) * T.lda];
      a[q] = v;
    }
#pragma unroll
    for (int q = 0; q < EB; ++q) {
      const int e = tid + q * kThreads;
      int j, kk;
      if (!tb) { kk = e % BK; j = e / BK; } else { j = e % BN; kk = e / BN; }
      const int gj = col0 + j;
      V v = zero();
      if (gj < J.n && kk < kt) v = tb ? B[gj + (long long)(k0 + kk) * T.ldb] : B[(k0 + kk) + (long long)gj * T.ldb];
      b[q] = v;
    }
  }
  static __device__ __forceinline__ V zero() {
    if constexpr (std::is_same<V, double2>::value) return make_double2(0.0, 0.0);
    else return 0.0;
  }
  // index helpers for the shared-memory store of element q
  static __device__ __forceinline__ void a_pos(bool ta, int q, int& i, int& kk) {
    const int e = threadIdx.x + q * kThreads;
    if (!ta) { i = e % BM; kk = e / BM; } else { kk = e % BK; i = e / BK; }
  }
  static __device__ __forceinline__ void b_pos(bool tb, int q, int& j, int& kk) {
    const int e = threadIdx.x + q * kThreads;
    if (!tb) { kk = e % BK; j = e / BK; } else { j = e % BN; kk = e / BN; }
  }
};

// ---------------------------------------------------------------------------
// Split-K fixup, run by every thread of an item that wrote a partial tile: the
// last item of the tile to finish (per-tile atomic count) sums all its partial
// tiles in slot order -- the same order whichever item is last -- adds C when
// the job accumulates, writes C and clears the count for the next launch.
template <bool CPLX>
__device__ void split_fixup(const WorkItem& it, const GemmJob& J, const RedItem* __restrict__ reds,
                            const Bases& bases, const void* work, int* tile_cnt, int BM, int BN) {
  __shared__ int last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&tile_cnt[it.red], 1) == reds[it.red].nslot - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const RedItem R = reds[it.red];
  const int row0 = R.tm * BM, col0 = R.tn * BN;
  const bool accum = J.flags & JF_ACCUM;
  for (int e = threadIdx.x; e < BM * BN; e += blockDim.x) {
    const int r = e % BM, c = e / BM;
    if (row0 + r >= J.m || col0 + c >= J.n) continue;
    const long long idx = (row0 + r) + (long long)(col0 + c) * J.ldc;
    if (CPLX) {
      const double2* W = static_cast<const double2*>(work);
      double2 sum = make_double2(0.0, 0.0);
      for (int k = 0; k < R.nslot; ++k) {
        const double2 v = __ldcg(W + (long long)(R.slot0 + k) * BM * BN + e);
        sum.x += v.x;
        sum.y += v.y;
      }
      double2* C = static_cast<double2*>(bases.p[J.cbuf]) + J.coff;
      if (accum) { const double2 o = C[idx]; sum.x += o.x; sum.y += o.y; }
      C[idx] = sum;
    } else {
      const double* W = static_cast<const double*>(work);
      double sum = 0.0;
      for (int k = 0; k < R.nslot; ++k) sum += __ldcg(W + (long long)(R.slot0 + k) * BM * BN + e);
      double* C = static_cast<double*>(bases.p[J.cbuf]) + J.coff;
      C[idx] = accum ? C[idx] + sum : sum;
    }
  }
  if (threadIdx.x == 0) tile_cnt[it.red] = 0;
}

// ---------------------------------------------------------------------------
// FP64, real, multistage: slabs are copied global -> shared with cp.async (8-byte,
// zero-filled outside the block), STAGES-1 slabs in flight while the tensor cores
// consume one.  Each operand slab is kept in the layout its global copy is
// contiguous in (k-major for A, n-major for B when not transposed; the other way
// when transposed), and the fragment loads follow that layout; row strides of
// 68 / 20 doubles keep both the copies and the fragment loads conflict free.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int BM, int BN, int BK, int STAGES>
__global__ void __launch_bounds__(kThreads, 3) items_f64_ms(const GemmTerm* __restrict__ terms,
                                                            const GemmJob* __restrict__ jobs,
                                                            const WorkItem* __restrict__ items, Bases bases,
                                                            double* __restrict__ work,
                                                            const RedItem* __restrict__ reds, int* tile_cnt, const int* mask) {
  static_assert(BM == 64 && BN == 64 && BK == 16, "layout strides assume 64 x 64 x 16");
  constexpr int SK = BM + 4;        // k-major row stride (rows of m or n)
  constexpr int SM = BK + 4;        // m/n-major row stride (rows of k)
  constexpr int ABUF = (BM * SM > BK * SK) ? BM * SM : BK * SK;
  constexpr int BBUF = (BN * SM > BK * SK) ? BN * SM : BK * SK;
  extern __shared__ __align__(16) double smem_ms[];
  double* As = smem_ms;                         // STAGES x ABUF
  double* Bs = smem_ms + STAGES * ABUF;         // STAGES x BBUF
  __shared__ double sh_alpha[STAGES];
  __shared__ int sh_flags[STAGES];
  const WorkItem it = items[blockIdx.x];
  const GemmJob J = jobs[it.job];
  if (mask && !mask[J.tag]) return;   // instance switched off for this launch
  const int row0 = it.tm * BM, col0 = it.tn * BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  constexpr int WM = BM / 2, WN = BN / 2, MT = WM / 8, NT = WN / 8;
  constexpr int EA = BM * BK / kThreads, EB = BK * BN / kThreads;
  double acc[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  SlabWalk w{J.t0 + it.t0, it.k0, it.kcount};

  auto issue = [&](int st, int tt, int k0, int kt) {
    const GemmTerm T = terms[tt];
    const bool ta = T.flags & TF_TA, tb = T.flags & TF_TB;
    const double* A = static_cast<const double*>(bases.p[T.abuf]) + T.aoff;
    const double* B = static_cast<const double*>(bases.p[T.bbuf]) + T.boff;
    double* as = As + st * ABUF;
    double* bs = Bs + st * BBUF;
#pragma unroll
    for (int q = 0; q < EA; ++q) {
      const int e = tid + q * kThreads;
      int i, kk;
      if (!ta) { i = e % BM; kk = e / BM; } else { kk = e % BK; i = e / BK; }
      const int gi = row0 + i;
      const bool ok = gi < J.m && kk < kt;
      const double* src = ok ? (ta ? A + (k0 + kk) + (long long)gi * T.lda : A + gi + (long long)(k0 + kk) * T.lda) : A;
      cp_async8(ta ? as + i * SM + kk : as + kk * SK + i, src, ok);
    }
#pragma unroll
    for (int q = 0; q < EB; ++q) {
      const int e = tid + q * kThreads;
      int j, kk;
      if (!tb) { kk = e % BK; j = e / BK; } else { j = e % BN; kk = e / BN; }
      const int gj = col0 + j;
      const bool ok = gj < J.n && kk < kt;
      const double* src = ok ? (tb ? B + gj + (long long)(k0 + kk) * T.ldb : B + (k0 + kk) + (long long)gj * T.ldb) : B;
      cp_async8(tb ? bs + kk * SK + j : bs + j * SM + kk, src, ok);
    }
    if (tid == 0) { sh_alpha[st] = T.ar; sh_flags[st] = T.flags; }
  };

  int issued = 0;
#pragma unroll
  for (int st = 0; st < STAGES - 1; ++st) {
    int tt, kk, kt;
    if (w.next(terms, BK, tt, kk, kt)) { issue(st, tt, kk, kt); ++issued; }
    cp_async_commit();
  }
  for (int c = 0; c < issued; ++c) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int st = c % STAGES;
    const double alpha = sh_alpha[st];
    const int fl = sh_flags[st];
    const bool ta = fl & TF_TA, tb = fl & TF_TB;
    const double* as = As + st * ABUF;
    const double* bs = Bs + st * BBUF;
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      const int k = k4 + (lane & 3);
      double af[MT], bf[NT];
#pragma unroll
      for (int mi = 0; mi < MT; ++mi) {
        const int r = wm * WM + mi * 8 + (lane >> 2);
        af[mi] = (ta ? as[r * SM + k] : as[k * SK + r]) * alpha;
      }
#pragma unroll
      for (int ni = 0; ni < NT; ++ni) {
        const int cc = wn * WN + ni * 8 + (lane >> 2);
        bf[ni] = tb ? bs[k * SK + cc] : bs[cc * SM + k];
      }
#pragma unroll
      for (int mi = 0; mi < MT; ++mi)
#pragma unroll
        for (int ni = 0; ni < NT; ++ni) dmma884(acc[mi][ni][0], acc[mi][ni][1], af[mi], bf[ni]);
    }
    int tt, kk, kt;
    if (w.next(terms, BK, tt, kk, kt)) { issue((c + STAGES - 1) % STAGES, tt, kk, kt); ++issued; }
    cp_async_commit();
  }
  cp_async_wait<0>();
  const bool direct = it.slot < 0;
  double* C = direct ? static_cast<double*>(bases.p[J.cbuf]) + J.coff : work + (long long)it.slot * BM * BN;
  const bool accum = J.flags & JF_ACCUM;
#pragma unroll
  for (int mi = 0; mi < MT; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = wm * WM + mi * 8 + (lane >> 2);
        const int c = wn * WN + ni * 8 + 2 * (lane & 3) + e;
        if (direct) {
          if (row0 + r < J.m && col0 + c < J.n) {
            const long long idx = (row0 + r) + (long long)(col0 + c) * J.ldc;
            C[idx] = accum ? C[idx] + acc[mi][ni][e] : acc[mi][ni][e];
          }
        } else {
          C[r + c * BM] = acc[mi][ni][e];
        }
      }
  if (it.slot >= 0) split_fixup<false>(it, J, reds, bases, work, tile_cnt, BM, BN);
}
constexpr int kF64Stages = 3;
constexpr size_t kF64MsSmem = (size_t)kF64Stages * 2 * (64 * 20) * sizeof(double);


// 3xTF32, real, multistage: the same FP64 slabs as items_f64_ms; operands are
// rounded to FP32 and split into TF32 hi/lo while the fragments are read.
template <int BM, int BN, int BK, int STAGES>
__global__ void __launch_bounds__(kThreads, 3) items_tf32x3_ms(const GemmTerm* __restrict__ terms,
                                                               const GemmJob* __restrict__ jobs,
                                                               const WorkItem* __restrict__ items, Bases bases,
                                                               double* __restrict__ work,
                                                               const RedItem* __restrict__ reds, int* tile_cnt, const int* mask) {
  static_assert(BM == 64 && BN == 64 && BK == 16, "layout strides assume 64 x 64 x 16");
  constexpr int SK = BM + 4, SM = BK + 4;
  constexpr int ABUF = (BM * SM > BK * SK) ? BM * SM : BK * SK;
  constexpr int BBUF = (BN * SM > BK * SK) ? BN * SM : BK * SK;
  extern __shared__ __align__(16) double smem_ms[];
  double* As = smem_ms;
  double* Bs = smem_ms + STAGES * ABUF;
  __shared__ double sh_alpha[STAGES];
  __shared__ int sh_flags[STAGES];
  const WorkItem it = items[blockIdx.x];
  const GemmJob J = jobs[it.job];
  if (mask && !mask[J.tag]) return;   // instance switched off for this launch
  const int row0 = it.tm * BM, col0 = it.tn * BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int g = lane >> 2, tg = lane & 3;
  constexpr int WM = BM / 2, WN = BN / 2, MT = WM / 16, NT = WN / 8;
  constexpr int EA = BM * BK / kThreads, EB = BK * BN / kThreads;
  double accd[MT][NT][4];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) accd[i][j][e] = 0.0;
  SlabWalk w{J.t0 + it.t0, it.k0, it.kcount};
  auto issue = [&](int st, int tt, int k0, int kt) {
    const GemmTerm T = terms[tt];
    const bool ta = T.flags & TF_TA, tb = T.flags & TF_TB;
    const double* A = static_cast<const double*>(bases.p[T.abuf]) + T.aoff;
    const double* B = static_cast<const double*>(bases.p[T.bbuf]) + T.boff;
    double* as = As + st * ABUF;
    double* bs = Bs + st * BBUF;
#pragma unroll
    for (int q = 0; q < EA; ++q) {
      const int e = tid + q * kThreads;
      int i, kk;
      if (!ta) { i = e % BM; kk = e / BM; } else { kk = e % BK; i = e / BK; }
      const int gi = row0 + i;
      const bool ok = gi < J.m && kk < kt;
      const double* src = ok ? (ta ? A + (k0 + kk) + (long long)gi * T.lda : A + gi + (long long)(k0 + kk) * T.lda) : A;
      cp_async8(ta ? as + i * SM + kk : as + kk * SK + i, src, ok);
    }
#pragma unroll
    for (int q = 0; q < EB; ++q) {
      const int e = tid + q * kThreads;
      int j, kk;
      if (!tb) { kk = e % BK; j = e / BK; } else { j = e % BN; kk = e / BN; }
      const int gj = col0 + j;
      const bool ok = gj < J.n && kk < kt;
      const double* src = ok ? (tb ? B + gj + (long long)(k0 + kk) * T.ldb : B + (k0 + kk) + (long long)gj * T.ldb) : B;
      cp_async8(tb ? bs + kk * SK + j : bs + j * SM + kk, src, ok);
    }
    if (tid == 0) { sh_alpha[st] = T.ar; sh_flags[st] = T.flags; }
  };
  int issued = 0;
#pragma unroll
  for (int st = 0; st < STAGES - 1; ++st) {
    int tt, kk, kt;
    if (w.next(terms, BK, tt, kk, kt)) { issue(st, tt, kk, kt); ++issued; }
    cp_async_commit();
  }
  for (int c = 0; c < issued; ++c) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int st = c % STAGES;
    const double alpha = sh_alpha[st];
    const int fl = sh_flags[st];
    const bool ta = fl & TF_TA, tb = fl & TF_TB;
    const double* as = As + st * ABUF;
    const double* bs = Bs + st * BBUF;
    float acc[MT][NT][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
#pragma unroll
    for (int k8 = 0; k8 < BK; k8 += 8) {
      uint32_t ah[MT][4], al[MT][4], bh[NT][2], bl[NT][2];
#pragma unroll
      for (int mi = 0; mi < MT; ++mi) {
        const int r = wm * WM + mi * 16 + g;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int rr = r + ((e & 1) ? 8 : 0), k = k8 + tg + ((e & 2) ? 4 : 0);
          split3((ta ? as[rr * SM + k] : as[k * SK + rr]) * alpha, ah[mi][e], al[mi][e]);
        }
      }
#pragma unroll
      for (int ni = 0; ni < NT; ++ni) {
        const int cc = wn * WN + ni * 8 + g;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int k = k8 + tg + (e ? 4 : 0);
          split3(tb ? bs[k * SK + cc] : bs[cc * SM + k], bh[ni][e], bl[ni][e]);
        }
      }
#pragma unroll
      for (int mi = 0; mi < MT; ++mi)
#pragma unroll
        for (int ni = 0; ni < NT; ++ni) {
          mma_tf32(acc[mi][ni], al[mi], bh[ni]);
          mma_tf32(acc[mi][ni], ah[mi], bl[ni]);
          mma_tf32(acc[mi][ni], ah[mi], bh[ni]);
        }
    }
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) accd[i][j][e] += (double)acc[i][j][e];
    int tt, kk, kt;
    if (w.next(terms, BK, tt, kk, kt)) { issue((c + STAGES - 1) % STAGES, tt, kk, kt); ++issued; }
    cp_async_commit();
  }
  cp_async_wait<0>();
  const bool direct = it.slot < 0;
  double* C = direct ? static_cast<double*>(bases.p[J.cbuf]) + J.coff : work + (long long)it.slot * BM * BN;
  const bool accum = J.flags & JF_ACCUM;
#pragma unroll
  for (int mi = 0; mi < MT; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = wm * WM + mi * 16 + g + (e >= 2 ? 8 : 0);
        const int c = wn * WN + ni * 8 + 2 * tg + (e & 1);
        if (direct) {
          if (row0 + r < J.m && col0 + c < J.n) {
            const long long idx = (row0 + r) + (long long)(col0 + c) * J.ldc;
            C[idx] = accum ? C[idx] + accd[mi][ni][e] : accd[mi][ni][e];
          }
        } else {
          C[r + c * BM] = accd[mi][ni][e];
        }
      }
  if (it.slot >= 0) split_fixup<false>(it, J, reds, bases, work, tile_cnt, BM, BN);
}

// ---------------------------------------------------------------------------
// FP64, complex: rr = Re*Re, ii = Im*Im, im = Re*Im + Im*Re; C = rr - ii + i im
template <int BM, int BN, int BK>
__global__ void __launch_bounds__(kThreads) items_z64(const GemmTerm* __restrict__ terms, const GemmJob* __restrict__ jobs,
                                                      const WorkItem* __restrict__ items, Bases bases,
                                                      double2* __restrict__ work, const RedItem* __restrict__ reds,
                                                      int* tile_cnt, const int* mask) {
  constexpr int PAD = 4;
  __shared__ double Ar[2][BK][BM + PAD], Ai[2][BK][BM + PAD];
  __shared__ double Br[2][BK][BN + PAD], Bi[2][BK][BN + PAD];
  using SL = Slab<double2, BM, BN, BK>;
  const WorkItem it = items[blockIdx.x];
  const GemmJob J = jobs[it.job];
  if (mask && !mask[J.tag]) return;   // instance switched off for this launch
  const int row0 = it.tm * BM, col0 = it.tn * BN;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  constexpr int WM = BM / 2, WN = BN / 2, MT = WM / 8, NT = WN / 8;
  double rr[MT][NT][2], ii[MT][NT][2], im[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) rr[i][j][e] = ii[i][j][e] = im[i][j][e] = 0.0;
  SlabWalk w{J.t0 + it.t0, it.k0, it.kcount};
  SL s;
  int tt, kk, kt;
  auto store = [&](int buf, const GemmTerm& T) {
    const bool ta = T.flags & TF_TA, tb = T.flags & TF_TB;
    const double ca = (T.flags & TF_CA) ? -1.0 : 1.0, cb = (T.flags & TF_CB) ? -1.0 : 1.0;
#pragma unroll
    for (int q = 0; q < SL::EA; ++q) {
      int i, k;
      SL::a_pos(ta, q, i, k);
      const double x = s.a[q].x, y = s.a[q].y * ca;
      Ar[buf][k][i] = x * T.ar - y * T.ai;
      Ai[buf][k][i] = x * T.ai + y * T.ar;
    }
#pragma unroll
    for (int q = 0; q < SL::EB; ++q) {
      int j, k;
      SL::b_pos(tb, q, j, k);
      Br[buf][k][j] = s.b[q].x;
      Bi[buf][k][j] = s.b[q].y * cb;
    }
  };
  int buf = 0;
  bool have = w.next(terms, BK, tt, kk, kt);
  if (have) {
    const GemmTerm T = terms[tt];
    s.load(T, J, row0, col0, kk, kt, bases);
    store(0, T);
  }
  __syncthreads();
  while (have) {
    int t2, k2, kt2;
    const bool more = w.next(terms, BK, t2, k2, kt2);
    GemmTerm T2;
    if (more) { T2 = terms[t2]; s.load(T2, J, row0, col0, k2, kt2, bases); }
#pragma unroll
    for (int k4 = 0; k4 < BK; k4 += 4) {
      double ar[MT], ai[MT], br[NT], bi[NT];
#pragma unroll
      for (int mi = 0; mi < MT; ++mi) {
        ar[mi] = Ar[buf][k4 + (lane & 3)][wm * WM + mi * 8 + (lane >> 2)];
        ai[mi] = Ai[buf][k4 + (lane & 3)][wm * WM + mi * 8 + (lane >> 2)];
      }
#pragma unroll
      for (int ni = 0; ni < NT; ++ni) {
        br[ni] = Br[buf][k4 + (lane & 3)][wn * WN + ni * 8 + (lane >> 2)];
        bi[ni] = Bi[buf][k4 + (lane & 3)][wn * WN + ni * 8 + (lane >> 2)];
      }
#pragma unroll
      for (int mi = 0; mi < MT; ++mi)
#pragma unroll
        for (int ni = 0; ni < NT; ++ni) {
          dmma884(rr[mi][ni][0], rr[mi][ni][1], ar[mi], br[ni]);
          dmma884(ii[mi][ni][0], ii[mi][ni][1], ai[mi], bi[ni]);
          dmma884(im[mi][ni][0], im[mi][ni][1], ar[mi], bi[ni]);
          dmma884(im[mi][ni][0], im[mi][ni][1], ai[mi], br[ni]);
        }
    }
    if (more) store(buf ^ 1, T2);
    __syncthreads();
    buf ^= 1;
    have = more;
  }
  const bool direct = it.slot < 0;
  double2* C = direct ? static_cast<double2*>(bases.p[J.cbuf]) + J.coff : work + (long long)it.slot * BM * BN;
  const bool accum = J.flags & JF_ACCUM;
#pragma unroll
  for (int mi = 0; mi < MT; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = wm * WM + mi * 8 + (lane >> 2);
        const int c = wn * WN + ni * 8 + 2 * (lane & 3) + e;
        double2 v = make_double2(rr[mi][ni][e] - ii[mi][ni][e], im[mi][ni][e]);
        if (direct) {
          if (row0 + r < J.m && col0 + c < J.n) {
            const long long idx = (row0 + r) + (long long)(col0 + c) * J.ldc;
            if (accum) { const double2 o = C[idx]; v.x += o.x; v.y += o.y; }
            C[idx] = v;
          }
        } else {
          C[r + c * BM] = v;
        }
      }
  if (it.slot >= 0) split_fixup<true>(it, J, reds, bases, work, tile_cnt, BM, BN);
}

// ---------------------------------------------------------------------------
// 3xTF32 (real and complex), hi/lo planes in shared memory
template <bool CPLX, int BM, int BN, int BK>
__global__ void __launch_bounds__(kThreads) items_tf32x3(const GemmTerm* __restrict__ terms,
                                                         const GemmJob* __restrict__ jobs,
                                                         const WorkItem* __restrict__ items, Bases bases,
                                                         void* __restrict__ work, const RedItem* __restrict__ reds,
                                                         int* tile_cnt, const int* mask) {
  constexpr int PAD = 8;
  constexpr int NP = CPLX ? 2 : 1;
  using V = typename std::conditional<CPLX, double2, double>::type;
  using SL = Slab<V, BM, BN, BK>;
  __shared__ uint32_t Ah[2][NP][BK][BM + PAD], Al[2][NP][BK][BM + PAD];
  __shared__ uint32_t Bh[2][NP][BK][BN + PAD], Bl[2][NP][BK][BN + PAD];
  const WorkItem it = items[blockIdx.x];
  const GemmJob J = jobs[it.job];
  if (mask && !mask[J.tag]) return;   // instance switched off for this launch
  const int row0 = it.tm * BM, col0 = it.tn * BN;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int g = lane >> 2, tg = lane & 3;
  constexpr int WM = BM / 2, WN = BN / 2, MT = WM / 16, NT = WN / 8;
  constexpr int NACC = CPLX ? 3 : 1;
  double accd[NACC][MT][NT][4];
#pragma unroll
  for (int q = 0; q < NACC; ++q)
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) accd[q][i][j][e] = 0.0;
  SlabWalk w{J.t0 + it.t0, it.k0, it.kcount};
  SL s;
  int tt, kk, kt;
  auto store = [&](int buf, const GemmTerm& T) {
    const bool ta = T.flags & TF_TA, tb = T.flags & TF_TB;
    const double ca = (T.flags & TF_CA) ? -1.0 : 1.0, cb = (T.flags & TF_CB) ? -1.0 : 1.0;
#pragma unroll
    for (int q = 0; q < SL::EA; ++q) {
      int i, k;
      SL::a_pos(ta, q, i, k);
      if constexpr (CPLX) {
        const double x = s.a[q].x, y = s.a[q].y * ca;
        split3(x * T.ar - y * T.ai, Ah[buf][0][k][i], Al[buf][0][k][i]);
        split3(x * T.ai + y * T.ar, Ah[buf][NP - 1][k][i], Al[buf][NP - 1][k][i]);
      } else {
        split3(s.a[q] * T.ar, Ah[buf][0][k][i], Al[buf][0][k][i]);
      }
    }
#pragma unroll
    for (int q = 0; q < SL::EB; ++q) {
      int j, k;
      SL::b_pos(tb, q, j, k);
      if constexpr (CPLX) {
        split3(s.b[q].x, Bh[buf][0][k][j], Bl[buf][0][k][j]);
        split3(s.b[q].y * cb, Bh[buf][NP - 1][k][j], Bl[buf][NP - 1][k][j]);
      } else {
        split3(s.b[q], Bh[buf][0][k][j], Bl[buf][0][k][j]);
      }
    }
  };
  int buf = 0;
  bool have = w.next(terms, BK, tt, kk, kt);
  if (have) {
    const GemmTerm T = terms[tt];
    s.load(T, J, row0, col0, kk, kt, bases);
    store(0, T);
  }
  __syncthreads();
  while (have) {
    int t2, k2, kt2;
    const bool more = w.next(terms, BK, t2, k2, kt2);
    GemmTerm T2;
    if (more) { T2 = terms[t2]; s.load(T2, J, row0, col0, k2, kt2, bases); }
    float acc[NACC][MT][NT][4];
#pragma unroll
    for (int q = 0; q < NACC; ++q)
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) acc[q][i][j][e] = 0.f;
#pragma unroll
    for (int k8 = 0; k8 < BK; k8 += 8) {
      uint32_t ah[NP][MT][4], al[NP][MT][4], bh[NP][NT][2], bl[NP][NT][2];
#pragma unroll
      for (int p = 0; p < NP; ++p) {
#pragma unroll
        for (int mi = 0; mi < MT; ++mi) {
          const int r = wm * WM + mi * 16 + g;
          ah[p][mi][0] = Ah[buf][p][k8 + tg][r];         al[p][mi][0] = Al[buf][p][k8 + tg][r];
          ah[p][mi][1] = Ah[buf][p][k8 + tg][r + 8];     al[p][mi][1] = Al[buf][p][k8 + tg][r + 8];
          ah[p][mi][2] = Ah[buf][p][k8 + tg + 4][r];     al[p][mi][2] = Al[buf][p][k8 + tg + 4][r];
          ah[p][mi][3] = Ah[buf][p][k8 + tg + 4][r + 8]; al[p][mi][3] = Al[buf][p][k8 + tg + 4][r + 8];
        }
#pragma unroll
        for (int ni = 0; ni < NT; ++ni) {
          const int c = wn * WN + ni * 8 + g;
          bh[p][ni][0] = Bh[buf][p][k8 + tg][c];     bl[p][ni][0] = Bl[buf][p][k8 + tg][c];
          bh[p][ni][1] = Bh[buf][p][k8 + tg + 4][c]; bl[p][ni][1] = Bl[buf][p][k8 + tg + 4][c];
        }
      }
#pragma unroll
      for (int mi = 0; mi < MT; ++mi)
#pragma unroll
        for (int ni = 0; ni < NT; ++ni) {
          if constexpr (CPLX) {
            mma_tf32(acc[0][mi][ni], al[0][mi], bh[0][ni]);
            mma_tf32(acc[0][mi][ni], ah[0][mi], bl[0][ni]);
            mma_tf32(acc[0][mi][ni], ah[0][mi], bh[0][ni]);
            mma_tf32(acc[1][mi][ni], al[1][mi], bh[1][ni]);
            mma_tf32(acc[1][mi][ni], ah[1][mi], bl[1][ni]);
            mma_tf32(acc[1][mi][ni], ah[1][mi], bh[1][ni]);
            mma_tf32(acc[2][mi][ni], al[0][mi], bh[1][ni]);
            mma_tf32(acc[2][mi][ni], ah[0][mi], bl[1][ni]);
            mma_tf32(acc[2][mi][ni], ah[0][mi], bh[1][ni]);
            mma_tf32(acc[2][mi][ni], al[1][mi], bh[0][ni]);
            mma_tf32(acc[2][mi][ni], ah[1][mi], bl[0][ni]);
            mma_tf32(acc[2][mi][ni], ah[1][mi], bh[0][ni]);
          } else {
            mma_tf32(acc[0][mi][ni], al[0][mi], bh[0][ni]);
            mma_tf32(acc[0][mi][ni], ah[0][mi], bl[0][ni]);
            mma_tf32(acc[0][mi][ni], ah[0][mi], bh[0][ni]);
          }
        }
    }
#pragma unroll
    for (int q = 0; q < NACC; ++q)
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) accd[q][i][j][e] += (double)acc[q][i][j][e];
    if (more) store(buf ^ 1, T2);
    __syncthreads();
    buf ^= 1;
    have = more;
  }
  const bool direct = it.slot < 0;
  const bool accum = J.flags & JF_ACCUM;
#pragma unroll
  for (int mi = 0; mi < MT; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = wm * WM + mi * 16 + g + (e >= 2 ? 8 : 0);
        const int c = wn * WN + ni * 8 + 2 * tg + (e & 1);
        if constexpr (CPLX) {
          double2 v = make_double2(accd[0][mi][ni][e] - accd[1][mi][ni][e], accd[NACC - 1][mi][ni][e]);
          if (direct) {
            if (row0 + r < J.m && col0 + c < J.n) {
              double2* C = static_cast<double2*>(bases.p[J.cbuf]) + J.coff;
              const long long idx = (row0 + r) + (long long)(col0 + c) * J.ldc;
              if (accum) { const double2 o = C[idx]; v.x += o.x; v.y += o.y; }
              C[idx] = v;
            }
          } else {
            static_cast<double2*>(work)[(long long)it.slot * BM * BN + r + c * BM] = v;
          }
        } else {
          const double v = accd[0][mi][ni][e];
          if (direct) {
            if (row0 + r < J.m && col0 + c < J.n) {
              double* C = static_cast<double*>(bases.p[J.cbuf]) + J.coff;
              const long long idx = (row0 + r) + (long long)(col0 + c) * J.ldc;
              C[idx] = accum ? C[idx] + v : v;
            }
          } else {
            static_cast<double*>(work)[(long long)it.slot * BM * BN + r + c * BM] = v;
          }
        }
      }
  if (it.slot >= 0) split_fixup<CPLX>(it, J, reds, bases, work, tile_cnt, BM, BN);
}

int gemm_tile_m(bool cplx, int /*prec*/) { return cplx ? 32 : 64; }
int gemm_tile_n(bool cplx, int /*prec*/) { return cplx ? 32 : 64; }

void launch_items(bool cplx, int prec, const GemmTerm* terms, const GemmJob* jobs, const WorkItem* items, int nitems,
                  const Bases& b, void* work, const RedItem* reds, int* tile_cnt, const int* mask,
                  cudaStream_t s) {
  if (nitems <= 0) return;
  if (prec == PREC_TF32X3) {
    if (cplx) {
      items_tf32x3<true, 32, 32, 16><<<nitems, kThreads, 0, s>>>(terms, jobs, items, b, work, reds, tile_cnt, mask);
    } else {
      static unsigned char attr[kMaxDevices] = {0};
      ensure_smem_attr((const void*)items_tf32x3_ms<64, 64, 16, kF64Stages>, (int)kF64MsSmem, attr);
      items_tf32x3_ms<64, 64, 16, kF64Stages><<<nitems, kThreads, kF64MsSmem, s>>>(terms, jobs, items, b,
                                                                                 static_cast<double*>(work), reds,
                                                                                 tile_cnt, mask);
    }
  } else {
    if (cplx) {
      items_z64<32, 32, 16><<<nitems, kThreads, 0, s>>>(terms, jobs, items, b, static_cast<double2*>(work), reds,
                                                          tile_cnt, mask);
    } else {
      static unsigned char attr[kMaxDevices] = {0};
      ensure_smem_attr((const void*)items_f64_ms<64, 64, 16, kF64Stages>, (int)kF64MsSmem, attr);
      items_f64_ms<64, 64, 16, kF64Stages><<<nitems, kThreads, kF64MsSmem, s>>>(terms, jobs, items, b,
                                                                              static_cast<double*>(work), reds,
                                                                              tile_cnt, mask);
    }
  }
}

// ---------------------------------------------------------------------------
// Fixed scratch for the allocation-free H_eff*psi entry point.  It lives for the
// life of the process on every device that loads the library.  Host code must not
// use the symbol's host-side name as a device address: the device address is
// looked up once per device with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

int noalloc_scratch(void** ptr) {
  static std::mutex mu;
  static void* cache[kMaxDevices] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kMaxDevices) return (int)cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(mu);
  if (!cache[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return (int)e;
    cache[dev] = p;
  }
  *ptr = cache[dev];
  return 0;
}


}  // namespace sadmrg
