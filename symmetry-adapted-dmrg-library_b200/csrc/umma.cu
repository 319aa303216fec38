// umma.cu -- 3xTF32 grouped block-GEMM on the fifth-generation tensor cores
// (tcgen05.mma .kind::tf32, FP32 accumulators in tensor memory); complex plans
// run in the real form described in kernels.cuh.
//
// Operands are pre-split into TF32 hi/lo panels (layout in kernels.cuh): the
// constant operators once per plan, psi once per matvec (pack_kernel), and the
// intermediate X = op1^T psi directly by the epilogue of the stage that makes
// it.  The GEMM then does no per-element work in its main loop:
//
//   warp 0 (one lane)  producer: per slab, two cp.async.bulk copies (A panel
//                      128 x 32, B panel BN x 32, hi + lo) into a ring of
//                      shared-memory stages, completion tracked by the stage's
//                      mbarrier (expect_tx);
//   warp 1 (one lane)  issuer: per 8-wide k step three tcgen05.mma (lo*hi,
//                      hi*lo, hi*hi) into the item's accumulator; tcgen05.commit
//                      frees the stage, and after the item's last slab signals
//                      the accumulator full;
//   warps 2-5          epilogue: tcgen05.ld of the 128 x BN accumulator (each
//                      warp its 32 lanes), then FP64 store (optionally adding)
//                      or hi/lo panels of X; a split-K item writes an FP32
//                      partial tile and the last item of its tile to finish
//                      (atomic count per tile) sums all partials in slot order.
// Two accumulators (2 x BN TMEM columns) let the epilogue of one item overlap
// the MMAs of the next; the kernel is persistent (one CTA per SM -- or two,
// with a 2-stage ring each, at tile width 64 -- static round-robin over the
// longest-first item list).
//
// Every mbarrier wait is bounded (time and iterations) and also gives up when
// another role has failed.  A wait that runs out sets a device status word
// (umma_status) and the CTA stops; before it frees its tensor memory and exits
// it waits, again bounded, for the copies and MMAs it issued.
#include <cuda_runtime.h>
#include <cstdint>

#include "kernels.cuh"

namespace sadmrg {
namespace {

constexpr unsigned long long kWaitNs = 2000000000ull;   // 2 s per wait
constexpr long long kWaitIters = 1ll << 26;
constexpr int kGThreads = 192;                          // 6 warps: producer, issuer, 4 x epilogue

__device__ int g_umma_status = 0;

__device__ __forceinline__ uint32_t saddr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}
// x ~ hi + lo, both TF32 (the split of the mma.sync 3xTF32 path)
__device__ __forceinline__ void split_hl(double v, uint32_t& hi, uint32_t& lo) {
  const float f = (float)v;
  hi = tf32_rna(f);
  lo = tf32_rna(f - __uint_as_float(hi));
}
__device__ __forceinline__ void split_hl_f(float f, uint32_t& hi, uint32_t& lo) {
  hi = tf32_rna(f);
  lo = tf32_rna(f - __uint_as_float(hi));
}

// shared-memory matrix descriptor: K-major, no swizzle, version 1
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor, kind::tf32: D f32, A/B tf32, both K-major, M x N
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(da), "l"(db), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
// one contiguous global -> shared copy, completion counted on the mbarrier (no multicast)
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Bounded wait for the phase with the given parity.  Gives up (false) after
// limit_ns, or as soon as *abort is set when abort is non-null.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const volatile int* abort,
                                          unsigned long long limit_ns = kWaitNs) {
  const unsigned long long t0 = gtime();
  for (long long i = 0; i < kWaitIters; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((i & 63) == 63) {
      if (abort && *abort) return false;
      if (gtime() - t0 > limit_ns) return false;
    }
  }
  return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

__device__ __forceinline__ void st_global_v4(void* p, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
  *reinterpret_cast<uint4*>(p) = make_uint4(x, y, z, w);
}

// ---------------------------------------------------------------------------
// FP64 matrices -> TF32 hi/lo panels.  One thread per 16-byte chunk (4 k of one
// row) -- of every row and k group of the padded panels, or (sparse jobs: psi,
// packed every matvec into panels zeroed when the plan was built) of the real rows
// and k only; consecutive threads take consecutive rows of one (slab, kg) column, so
// the stores are contiguous and the loads coalesce along rows (trans 0) or read
// one 32-byte sector per thread (trans 1).  Every job starts on a multiple of
// 256 chunks, so a block works for one job, looked up in blk_job.
__device__ __forceinline__ void pack_chunk(const PackJob& P, unsigned local, const Bases& bases,
                                           unsigned char* __restrict__ dst) {
  const unsigned T = (unsigned)P.T;
  const unsigned nslab = ((unsigned)P.K + kPanelK - 1) / kPanelK;
  unsigned r, kgs;
  if (P.sparse) {
    const unsigned rows = (unsigned)P.rows;
    if (local >= rows * (((unsigned)P.K + 3u) / 4u)) return;
    r = local % rows;
    kgs = local / rows;
  } else {
    const unsigned Rp = (((unsigned)P.rows + T - 1) / T) * T;
    if (local >= Rp * nslab * 8u) return;
    r = local % Rp;
    kgs = local / Rp;
  }
  const unsigned s = kgs >> 3, kg = kgs & 7u;
  const unsigned p = r / T, rr = r - p * T;
  uint32_t h[4], l[4];
  if (P.cmode == 0) {
    const double* src = static_cast<const double*>(bases.p[P.srcbuf]) + P.src;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const unsigned k = s * kPanelK + kg * 4 + u;
      double v = 0.0;
      if (r < (unsigned)P.rows && k < (unsigned)P.K)
        v = P.trans ? src[k + (long long)r * P.ld] : src[r + (long long)k * P.ld];
      split_hl(v, h[u], l[u]);
    }
  } else {
    // real form of a complex operand: element (i, j) of op(src) feeds k = 2j, 2j + 1
    const double2* src = static_cast<const double2*>(bases.p[P.srcbuf]) + P.src;
    const unsigned i = P.cmode == 1 ? (r >> 1) : r, p1 = r & 1u;
#pragma unroll
    for (int u = 0; u < 4; u += 2) {
      const unsigned k = s * kPanelK + kg * 4 + u;   // even
      double2 z = make_double2(0.0, 0.0);
      if (r < (unsigned)P.rows && k < (unsigned)P.K) {
        const unsigned j = k >> 1;
        z = P.trans ? src[j + (long long)i * P.ld] : src[i + (long long)j * P.ld];
        if (P.conj) z.y = -z.y;
      }
      double v0, v1;
      if (P.cmode == 2) { v0 = z.x; v1 = z.y; }            // Bh(2j, l), Bh(2j + 1, l)
      else if (p1 == 0) { v0 = z.x; v1 = -z.y; }           // Ah(2i, 2j), Ah(2i, 2j + 1)
      else { v0 = z.y; v1 = z.x; }                         // Ah(2i + 1, 2j), Ah(2i + 1, 2j + 1)
      split_hl(v0, h[u], l[u]);
      split_hl(v1, h[u + 1], l[u + 1]);
    }
  }
  unsigned char* panel = dst + P.dst + ((long long)p * nslab + s) * (T * 256u);
  const unsigned off = (kg * T + rr) * 16u;
  st_global_v4(panel + off, h[0], h[1], h[2], h[3]);
  st_global_v4(panel + T * 128u + off, l[0], l[1], l[2], l[3]);
}

__global__ void __launch_bounds__(256) pack_kernel(const PackJob* __restrict__ jobs, const int* __restrict__ blk_job,
                                                   Bases bases, unsigned char* __restrict__ dst) {
  const PackJob P = jobs[blk_job[blockIdx.x]];
  pack_chunk(P, blockIdx.x * 256u + threadIdx.x - (unsigned)P.chunk0, bases, dst);
}

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// generic-proxy global writes <-> async-proxy (bulk copy) global reads
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// ---------------------------------------------------------------------------
template <int BN, int ST>
struct UG {
  static constexpr uint32_t ABYTES = kUmmaTileM * 256;   // A panel: hi + lo planes
  static constexpr uint32_t BBYTES = BN * 256;
  static constexpr uint32_t SBYTES = ABYTES + BBYTES;    // one stage
  static constexpr uint32_t SMEM = ST * SBYTES + 1024;
  static constexpr uint32_t TCOLS = 2 * BN;              // two accumulators
  static_assert(BN == 64 || BN == 128, "tile width");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

template <int BN, int ST, int MINB>
__global__ void __launch_bounds__(kGThreads, MINB)
    umma_gemm(const UTerm* __restrict__ terms, const UJob* __restrict__ jobs, const UItem* __restrict__ items,
              const URed* __restrict__ reds, int nitems, Bases bases, UBufs ub, UPhase ph) {
  using G = UG<BN, ST>;
  constexpr int BM = kUmmaTileM;
  extern __shared__ unsigned char usm_raw[];
  __shared__ __align__(8) unsigned long long full[ST], empty[ST], tfull[2], tempty[2];
  __shared__ uint32_t tmem_sh;
  __shared__ volatile int abort_sh;
  __shared__ volatile int last_sh;
  __shared__ volatile int ep_fail;
  __shared__ int pk_cnt[kMaxPackJobs];

  unsigned char* usm =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(usm_raw) + 127) & ~uintptr_t(127));
  const uint32_t sbase = saddr(usm);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned long long wlim = ph.wait_ns > 0 ? (unsigned long long)ph.wait_ns : kWaitNs;

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(&tmem_sh)),
                 "r"(G::TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    for (int i = 0; i < ST; ++i) {
      mbar_init(saddr(&full[i]), 1);
      mbar_init(saddr(&empty[i]), 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(saddr(&tfull[i]), 1);
      mbar_init(saddr(&tempty[i]), 4 * 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    abort_sh = 0;
    ep_fail = 0;
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_sh;

  if (ph.npk_blocks > 0) {
    // psi -> panels for this launch, by every thread: warps take 32-chunk groups
    // (a group never straddles two jobs, whose chunk ranges are multiples of 256),
    // count them per job in shared memory, then add each job's count once.
    for (int j = tid; j < ph.npk_jobs; j += kGThreads) pk_cnt[j] = 0;
    __syncthreads();
    const unsigned ngroups = (unsigned)ph.npk_blocks * 8u;
    for (unsigned gi = blockIdx.x * (kGThreads / 32) + warp; gi < ngroups; gi += gridDim.x * (kGThreads / 32)) {
      const int job = ph.pk_blk[gi >> 3];
      const PackJob P = ph.pk[job];
      pack_chunk(P, gi * 32u + (unsigned)lane - (unsigned)P.chunk0, bases, ub.pvar);
      if (lane == 0) atomicAdd(&pk_cnt[job], 32);
    }
    fence_proxy_async_global();
    __threadfence();
    __syncthreads();
    for (int j = tid; j < ph.npk_jobs; j += kGThreads)
      if (pk_cnt[j] > 0) atomicAdd(ub.deps + j, pk_cnt[j]);
  }

  if (warp == 0) {
    // ---------------- producer ----------------
    if (lane == 0) {
      long long g = 0;
      uint32_t last_bar = 0, last_par = 0;
      bool issued_any = false;
      int ready_term = -1;
      // bounded wait until dependency counter d reaches its target
      auto dep_wait = [&](int d) -> bool {
        if (d < 0) return true;
        const int target = ub.dep_target[d];
        const unsigned long long t0 = gtime();
        for (long long i = 0; i < kWaitIters; ++i) {
          if (ld_acquire(ub.deps + d) >= target) return true;
          if ((i & 63) == 63 && (abort_sh || gtime() - t0 > wlim)) return false;
          __nanosleep(64);
        }
        return false;
      };
      for (int ii = blockIdx.x; ii < nitems && !abort_sh; ii += gridDim.x) {
        const UItem it = items[ii];
        if (ub.mask && !ub.mask[jobs[it.job].tag]) continue;   // instance switched off for this launch
        int t = it.t0, s = it.s0;
        for (int q = 0; q < it.nslab; ++q) {
          while (s >= terms[t].nslab) { ++t; s = 0; }
          const UTerm T = terms[t];
          if (ph.wait_deps && t != ready_term) {
            // the panels this term reads are written in this launch: wait for them
            if (!dep_wait(T.adep) || !dep_wait(T.bdep)) {
              if (!abort_sh) atomicExch(&g_umma_status, 9);
              abort_sh = 1;
              break;
            }
            fence_proxy_async_global();
            ready_term = t;
          }
          const int st = (int)(g % ST);
          const uint32_t n = (uint32_t)(g / ST);
          if (!mbar_wait(saddr(&empty[st]), (n & 1u) ^ 1u, &abort_sh, wlim)) {
            if (!abort_sh) atomicExch(&g_umma_status, 3);
            abort_sh = 1;
            break;
          }
          const uint32_t fb = saddr(&full[st]);
          mbar_expect_tx(fb, G::SBYTES);
          const unsigned char* A = (T.abuf ? ub.pvar : ub.pconst) + T.a + ((long long)it.tm * T.nslab + s) * G::ABYTES;
          const unsigned char* B = (T.bbuf ? ub.pvar : ub.pconst) + T.b + ((long long)it.tn * T.nslab + s) * G::BBYTES;
          const uint32_t sa = sbase + (uint32_t)st * G::SBYTES;
          bulk_g2s(sa, A, G::ABYTES, fb);
          bulk_g2s(sa + G::ABYTES, B, G::BBYTES, fb);
          last_bar = fb;
          last_par = n & 1u;
          issued_any = true;
          ++g;
          ++s;
        }
      }
      // every copy this thread issued has landed before the CTA can exit: the last
      // copy into each stage (bulk copies may complete out of order, and after an
      // abort the issuer has not consumed them all)
      (void)last_bar;
      (void)last_par;
      if (issued_any)
        for (long long j = g > ST ? g - ST : 0; j < g; ++j)
          if (!mbar_wait(saddr(&full[(int)(j % ST)]), (uint32_t)(j / ST) & 1u, nullptr))
            atomicExch(&g_umma_status, 4);
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t idesc = tf32_idesc(BM, BN);
      long long g = 0;
      int il = 0;
      uint32_t last_bar = 0, last_par = 0;
      bool committed = false;
      for (int ii = blockIdx.x; ii < nitems && !abort_sh; ii += gridDim.x) {
        const UItem it = items[ii];
        if (ub.mask && !ub.mask[jobs[it.job].tag]) continue;
        const int acc = il & 1;
        if (!mbar_wait(saddr(&tempty[acc]), (((uint32_t)il >> 1) & 1u) ^ 1u, &abort_sh, wlim)) {
          if (!abort_sh) atomicExch(&g_umma_status, 5);
          abort_sh = 1;
          break;
        }
        fence_after();
        const uint32_t d = tmem + (uint32_t)(acc * BN);
        int t = it.t0, s = it.s0;
        bool ok = true;
        for (int q = 0; q < it.nslab; ++q) {
          while (s >= terms[t].nslab) { ++t; s = 0; }
          const UTerm T = terms[t];
          const int kt = (s == T.nslab - 1) ? T.klast : kPanelK;
          const int st = (int)(g % ST);
          const uint32_t n = (uint32_t)(g / ST);
          if (!mbar_wait(saddr(&full[st]), n & 1u, &abort_sh, wlim)) {
            if (!abort_sh) atomicExch(&g_umma_status, 6);
            abort_sh = 1;
            ok = false;
            break;
          }
          fence_after();
          const uint32_t a0 = sbase + (uint32_t)st * G::SBYTES, b0 = a0 + G::ABYTES;
          const int nks = (kt + 7) >> 3;
          for (int ks = 0; ks < nks; ++ks) {
            const uint32_t ao = (uint32_t)ks * 2u * BM * 16u, bo = (uint32_t)ks * 2u * BN * 16u;
            const uint64_t ah = kmajor_desc(a0 + ao, BM * 16, 128);
            const uint64_t al = kmajor_desc(a0 + BM * 128 + ao, BM * 16, 128);
            const uint64_t bh = kmajor_desc(b0 + bo, BN * 16, 128);
            const uint64_t bl = kmajor_desc(b0 + BN * 128 + bo, BN * 16, 128);
            umma_tf32(d, al, bh, idesc, (q > 0 || ks > 0) ? 1u : 0u);
            umma_tf32(d, ah, bl, idesc, 1u);
            umma_tf32(d, ah, bh, idesc, 1u);
          }
          umma_commit(saddr(&empty[st]));
          last_bar = saddr(&empty[st]);
          last_par = n & 1u;
          committed = true;
          ++g;
          ++s;
        }
        if (!ok) break;
        umma_commit(saddr(&tfull[acc]));
        last_bar = saddr(&tfull[acc]);
        last_par = ((uint32_t)il >> 1) & 1u;
        committed = true;
        ++il;
      }
      // every MMA this thread issued has finished before tensor memory is freed
      if (committed && !mbar_wait(last_bar, last_par, nullptr)) atomicExch(&g_umma_status, 7);
    }
  } else {
    // ---------------- epilogue: warps 2..5 ----------------
    const int quarter = warp & 3;           // TMEM lanes 32*quarter .. +31
    const int r = 32 * quarter + lane;      // tile row
    int il = 0;
    const int et = tid - 64;                // 0..127 within the epilogue warps
    // The four epilogue warps take every decision together: a failed wait is
    // posted to ep_fail and read by all after the same named barrier (id 1).
    for (int ii = blockIdx.x; ii < nitems; ii += gridDim.x) {
      const UItem it = items[ii];
      const UJob J = jobs[it.job];
      if (ub.mask && !ub.mask[J.tag]) continue;
      const int acc = il & 1;
      if (!mbar_wait(saddr(&tfull[acc]), ((uint32_t)il >> 1) & 1u, &abort_sh, wlim)) {
        if (!abort_sh) atomicExch(&g_umma_status, 8);
        abort_sh = 1;
        ep_fail = 1;
      }
      asm volatile("bar.sync 1, 128;" ::: "memory");
      if (ep_fail) break;
      fence_after();
      const int row0 = it.tm * BM, col0 = it.tn * BN;
      // 32 columns [cb, cb + 32) of row r of the finished tile -> C, or -> A panels of X
      auto emit = [&](int cb, const double (&x)[32]) {
        if (J.pack >= 0 && J.cx) {
          // real form Xh of the complex result: this thread holds Re (r even) or Im (r odd)
          // of row r/2, its lane neighbour the other part; columns [cb, cb + 32) feed
          // k = 2 (col0 + cb) .. + 63 of Xh, two slabs
          const bool odd = r & 1;
          const int s0 = 2 * (col0 + cb) / kPanelK;
#pragma unroll
          for (int hs = 0; hs < 2; ++hs) {
            const int s = s0 + hs;
            unsigned char* panel = ub.pvar + J.pack + ((long long)it.tm * J.pack_nslab + s) * (BM * 256);
            const bool live = s < J.pack_nslab;   // the same for every lane
#pragma unroll
            for (int kg = 0; kg < 8; ++kg) {
              uint32_t h[4], l[4];
#pragma unroll
              for (int w = 0; w < 2; ++w) {
                const int j = 16 * hs + 2 * kg + w;
                const double own = x[j];
                const double nb = __shfl_xor_sync(0xffffffffu, own, 1);
                const double v0 = own, v1 = odd ? nb : -nb;   // (Re, -Im) on row 2i, (Im, Re) on 2i + 1
                split_hl(J.alpha * v0, h[2 * w], l[2 * w]);
                split_hl(J.alpha * v1, h[2 * w + 1], l[2 * w + 1]);
              }
              if (live) {
                st_global_v4(panel + (kg * BM + r) * 16, h[0], h[1], h[2], h[3]);
                st_global_v4(panel + BM * 128 + (kg * BM + r) * 16, l[0], l[1], l[2], l[3]);
              }
            }
          }
        } else if (J.pack >= 0) {
          const int s = (col0 + cb) / kPanelK;
          if (s < J.pack_nslab) {
            unsigned char* panel = ub.pvar + J.pack + ((long long)it.tm * J.pack_nslab + s) * (BM * 256);
#pragma unroll
            for (int kg = 0; kg < 8; ++kg) {
              uint32_t h[4], l[4];
#pragma unroll
              for (int u = 0; u < 4; ++u) split_hl(J.alpha * x[4 * kg + u], h[u], l[u]);
              st_global_v4(panel + (kg * BM + r) * 16, h[0], h[1], h[2], h[3]);
              st_global_v4(panel + BM * 128 + (kg * BM + r) * 16, l[0], l[1], l[2], l[3]);
            }
          }
        } else if (row0 + r < J.m) {
          double* C = static_cast<double*>(bases.p[J.cbuf]) + J.coff;
          const bool accum = J.flags & JF_ACCUM;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = col0 + cb + j;
            if (col < J.n) {
              const long long idx = (row0 + r) + (long long)col * J.ldc;
              C[idx] = accum ? C[idx] + x[j] : x[j];
            }
          }
        }
      };
#pragma unroll 1
      for (int cb = 0; cb < BN; cb += 32) {
        uint32_t v[32];
        if (it.nslab > 0) {
          tmem_ld32(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)(acc * BN + cb), v);
        } else {
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] = 0u;
        }
        if (it.slot >= 0) {
          float* S = ub.slots + (long long)it.slot * BM * BN;
#pragma unroll
          for (int j = 0; j < 32; ++j) S[r + (cb + j) * BM] = __uint_as_float(v[j]);
        } else {
          double x[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) x[j] = (double)__uint_as_float(v[j]);
          emit(cb, x);
        }
      }
      fence_before();
      mbar_arrive(saddr(&tempty[acc]));
      // a finished tile of a result that later items read as panels: count it
      auto signal_tile = [&]() {
        if (J.dep < 0 || !ph.wait_deps) return;
        fence_proxy_async_global();
        __threadfence();
        asm volatile("bar.sync 1, 128;" ::: "memory");
        if (et == 0) atomicAdd(ub.deps + J.dep, 1);
      };
      if (it.slot < 0) signal_tile();
      if (it.slot >= 0) {
        // split-K: the last of the tile's items to get here sums every slot in
        // slot order (the same order whichever item is last) and emits the tile
        const URed R = reds[it.red];
        __threadfence();
        asm volatile("bar.sync 1, 128;" ::: "memory");
        if (tid == 64) last_sh = (atomicAdd(&ub.tile_cnt[it.red], 1) == R.nslot - 1) ? 1 : 0;
        asm volatile("bar.sync 1, 128;" ::: "memory");
        if (last_sh) {
          __threadfence();
#pragma unroll 1
          for (int cb = 0; cb < BN; cb += 32) {
            double x[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) x[j] = 0.0;
            for (int k = 0; k < R.nslot; ++k) {
              const float* S = ub.slots + (long long)(R.slot0 + k) * BM * BN;
#pragma unroll
              for (int j = 0; j < 32; ++j) x[j] += (double)__ldcg(S + r + (cb + j) * BM);
            }
            emit(cb, x);
          }
          if (tid == 64) ub.tile_cnt[it.red] = 0;   // ready for the next launch
        }
        asm volatile("bar.sync 1, 128;" ::: "memory");
        if (last_sh) signal_tile();
        asm volatile("bar.sync 1, 128;" ::: "memory");
      }
      ++il;
    }
  }

  fence_before();
  __syncthreads();
  if (warp == 1) {
    __syncwarp();
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(G::TCOLS) : "memory");
  }
  // the last CTA out clears the dependency counters for the next launch
  if (tid == 0 && ph.ndeps > 0) {
    __threadfence();
    if (atomicAdd(ub.fin, 1u) == gridDim.x - 1) {
      for (int d = 0; d < ph.ndeps; ++d) ub.deps[d] = 0;
      *ub.fin = 0u;
      __threadfence();
    }
  }
}

template <int BN, int ST, int MINB>
void launch_gemm_t(const UTerm* terms, const UJob* jobs, const UItem* items, const URed* reds, int nitems,
                   const Bases& b, const UBufs& u, const UPhase& ph, cudaStream_t s) {
  static unsigned char attr[kMaxDevices] = {0};
  static int occ[kMaxDevices] = {0};   // resident CTAs per SM the device grants this kernel
  ensure_smem_attr((const void*)umma_gemm<BN, ST, MINB>, (int)UG<BN, ST>::SMEM, attr);
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < kMaxDevices && occ[dev] == 0) {
    int v = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, umma_gemm<BN, ST, MINB>, kGThreads, UG<BN, ST>::SMEM) !=
            cudaSuccess || v < 1)
      v = 1;
    occ[dev] = v < MINB ? v : MINB;
  }
  const int per_sm = (dev >= 0 && dev < kMaxDevices) ? occ[dev] : 1;
  const int nsm = device_sm_count() * per_sm;   // CTAs resident at once
  int grid = nitems > ph.npk_blocks ? nitems : ph.npk_blocks;
  if (grid > nsm) grid = nsm;
  if (grid < 1) grid = 1;
  // CTAs wait on one another only when wait_deps is set: then every CTA must be
  // resident at once, which a cooperative launch guarantees
  if (ph.wait_deps) {
    Bases bb = b;
    UBufs uu = u;
    UPhase pp = ph;
    int ni = nitems;
    void* args[] = {(void*)&terms, (void*)&jobs, (void*)&items, (void*)&reds, (void*)&ni, (void*)&bb, (void*)&uu,
                    (void*)&pp};
    cudaLaunchCooperativeKernel((const void*)umma_gemm<BN, ST, MINB>, dim3(grid), dim3(kGThreads), args,
                                UG<BN, ST>::SMEM, s);
  } else {
    umma_gemm<BN, ST, MINB><<<grid, kGThreads, UG<BN, ST>::SMEM, s>>>(terms, jobs, items, reds, nitems, b, u, ph);
  }
}

}  // namespace

int device_sm_count() {
  static int n[kMaxDevices] = {0};
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
  if (n[dev] == 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) return 148;
    n[dev] = v;
  }
  return n[dev];
}

void ensure_smem_attr(const void* fn, int bytes, unsigned char* done) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return;
  }
  if (!done[dev]) {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    // the largest shared-memory carve-out, so that as many CTAs as the smem allows are resident
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
    done[dev] = 1;
  }
}

void launch_pack(const PackJob* jobs, const int* blk_job, int nblocks, const Bases& b, unsigned char* dst,
                 cudaStream_t s) {
  if (nblocks <= 0) return;
  pack_kernel<<<nblocks, 256, 0, s>>>(jobs, blk_job, b, dst);
}

void launch_umma_items(int bn, const UTerm* terms, const UJob* jobs, const UItem* items, const URed* reds, int nitems,
                       const Bases& b, const UBufs& u, const UPhase& ph, cudaStream_t s) {
  if (nitems <= 0 && ph.npk_blocks <= 0) return;
  if (bn == 128) launch_gemm_t<128, 3, 1>(terms, jobs, items, reds, nitems, b, u, ph, s);
  else if (ph.ctas_per_sm == 2) launch_gemm_t<64, 2, 2>(terms, jobs, items, reds, nitems, b, u, ph, s);
  else launch_gemm_t<64, 4, 1>(terms, jobs, items, reds, nitems, b, u, ph, s);
}

int umma_status(bool reset) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_umma_status, sizeof(int)) != cudaSuccess) return -1;
  if (reset && v != 0) {
    const int z = 0;
    cudaMemcpyToSymbol(g_umma_status, &z, sizeof(int));
  }
  return v;
}

}  // namespace sadmrg
