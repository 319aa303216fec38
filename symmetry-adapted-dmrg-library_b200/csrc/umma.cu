// umma.cu -- 3xTF32 grouped block-GEMM on the fifth-generation tensor cores
// (tcgen05.mma .kind::tf32, FP32 accumulator in tensor memory), real data.
//
// Same work-item contract as gemm.cu: an item is one output tile of a job and a
// contiguous range of the job's concatenated reduction dimension; an item that
// covers the whole range writes C (optionally accumulating), otherwise it writes
// its partial tile to a workspace slot that the fixed-order reduction sums.
// Output tiles are 128 x BN (one tcgen05.mma M=128, N=BN), k slabs are 32 wide.
//
// Per slab, 256 threads:
//   1. read the FP64 operands of the slab from global memory into registers
//      (one slab ahead, so the loads overlap the tensor-core work of the slab
//      before), coalesced along whichever index is contiguous in memory;
//   2. multiply A by the term's alpha, split every value into TF32 hi and lo
//      (x = hi + lo + O(2^-22 |x|)), and store four planes A_hi, A_lo, B_hi,
//      B_lo into shared memory in the K-major, no-swizzle core-matrix layout:
//      plane[kg][row][4] with kg = k / 4, i.e. 16-byte rows of 4 k values,
//      8-row core matrices 128 bytes apart (SBO), k halves of an 8-wide MMA
//      step R * 16 bytes apart (LBO);
//   3. one thread issues per 8-wide k step three tcgen05.mma (lo*hi, hi*lo,
//      hi*hi) into the same FP32 accumulator and commits them to the slab
//      buffer's mbarrier; two buffers, so step 2 of the next slab overlaps.
// Epilogue: each warp reads its 32 TMEM lanes x BN/2 columns with tcgen05.ld,
// widens to FP64 and stores (coalesced down each column).
//
// Every wait on an mbarrier is bounded (time and iterations).  A wait that runs
// out sets a device status word (read by umma_status), drains what this CTA
// issued (again bounded), frees its tensor memory and leaves the tile unwritten.
#include <cuda_runtime.h>
#include <cstdint>

#include "kernels.cuh"

namespace sadmrg {
namespace {

constexpr int kUBM = 128;             // tile rows = tcgen05.mma M
constexpr int kUBK = 32;              // k per slab
constexpr int kUThreads = 256;
constexpr unsigned long long kWaitNs = 2000000000ull;   // 2 s per wait
constexpr long long kWaitIters = 1ll << 26;

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
// x ~ hi + lo, both TF32 (the same split as the mma.sync 3xTF32 path)
__device__ __forceinline__ void split_hl(double v, uint32_t& hi, uint32_t& lo) {
  const float f = (float)v;
  hi = tf32_rna(f);
  lo = tf32_rna(f - __uint_as_float(hi));
}

__device__ __forceinline__ void st_shared_v4(uint32_t a, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(a), "r"(x), "r"(y), "r"(z), "r"(w) : "memory");
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
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

// bounded wait for the phase with the given parity; false if it ran out
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
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
    if ((i & 63) == 63 && gtime() - t0 > kWaitNs) break;
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

// Slab walk over an item's concatenated k (slabs never straddle a term).
struct UWalk {
  int t, k, rem;
  __device__ bool next(const GemmTerm* terms, int& tt, int& kk, int& kt) {
    if (rem <= 0) return false;
    int tk = terms[t].k;
    while (k >= tk) { ++t; k = 0; tk = terms[t].k; }
    tt = t;
    kk = k;
    kt = min(kUBK, min(tk - k, rem));
    k += kt;
    rem -= kt;
    return true;
  }
};

// Position (row, kg) of the q-th 16-byte chunk of this thread in an R-row plane.
// kcontig: k is the contiguous global index (a warp covers 8 rows x 4 chunks);
// otherwise the row index is (a warp covers 32 rows of one chunk column).
// Both give conflict-free 16-byte shared stores.
template <int R>
__device__ __forceinline__ void chunk_pos(bool kcontig, int q, int& row, int& kg) {
  const int e = (int)threadIdx.x + q * kUThreads;
  if (kcontig) {
    row = (e >> 2) % R;
    kg = (e & 3) + 4 * ((e >> 2) / R);
  } else {
    row = e % R;
    kg = e / R;
  }
}

template <int BN>
struct UCfg {
  static constexpr int KG = kUBK / 4;                        // 16-byte chunks along k
  static constexpr int APER = kUBM * KG / kUThreads;         // A chunks per thread
  static constexpr int BPER = BN * KG / kUThreads;           // B chunks per thread
  static constexpr uint32_t PA = kUBM * kUBK * 4;            // bytes of one A plane
  static constexpr uint32_t PB = BN * kUBK * 4;              // bytes of one B plane
  static constexpr uint32_t BUF = 2 * PA + 2 * PB;           // one slab buffer
  static constexpr uint32_t SMEM = 2 * BUF + 128;            // two buffers + alignment slack
  static constexpr uint32_t TCOLS = BN < 32 ? 32 : BN;       // TMEM columns (power of two >= 32)
  static_assert(APER * kUThreads == kUBM * KG && BPER * kUThreads == BN * KG, "chunk split");
  static_assert(BN == 64 || BN == 128, "tile width");
};

template <int BN>
__global__ void __launch_bounds__(kUThreads, 2)
    items_umma_tf32x3(const GemmTerm* __restrict__ terms, const GemmJob* __restrict__ jobs,
                      const WorkItem* __restrict__ items, Bases bases, double* __restrict__ work) {
  using C = UCfg<BN>;
  constexpr int BM = kUBM;
  extern __shared__ unsigned char usmem_raw[];
  __shared__ __align__(8) unsigned long long mbar[2];
  __shared__ uint32_t tmem_sh;
  __shared__ int abort_sh;

  unsigned char* usmem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(usmem_raw) + 127) & ~uintptr_t(127));
  const uint32_t sbase = saddr(usmem);
  const WorkItem it = items[blockIdx.x];
  const GemmJob J = jobs[it.job];
  const int row0 = it.tm * BM, col0 = it.tn * BN;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bar0 = saddr(&mbar[0]), bar1 = saddr(&mbar[1]);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(&tmem_sh)),
                 "r"(C::TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar1, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    abort_sh = 0;
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_sh;

  double ra[C::APER][4], rb[C::BPER][4];
  double s_alpha = 0.0;
  int s_flags = 0, s_kt = 0;

  auto load = [&](int tt, int k0, int kt) {
    const GemmTerm& T = terms[tt];
    const double* A = static_cast<const double*>(bases.p[T.abuf]) + T.aoff;
    const double* B = static_cast<const double*>(bases.p[T.bbuf]) + T.boff;
    const bool ta = T.flags & TF_TA, tb = T.flags & TF_TB;
    const int lda = T.lda, ldb = T.ldb;
#pragma unroll
    for (int q = 0; q < C::APER; ++q) {
      int row, kg;
      chunk_pos<BM>(ta, q, row, kg);
      const int gi = row0 + row;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int kk = 4 * kg + u;
        double v = 0.0;
        if (gi < J.m && kk < kt) v = ta ? A[(k0 + kk) + (long long)gi * lda] : A[gi + (long long)(k0 + kk) * lda];
        ra[q][u] = v;
      }
    }
#pragma unroll
    for (int q = 0; q < C::BPER; ++q) {
      int row, kg;
      chunk_pos<BN>(!tb, q, row, kg);
      const int gj = col0 + row;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int kk = 4 * kg + u;
        double v = 0.0;
        if (gj < J.n && kk < kt) v = tb ? B[gj + (long long)(k0 + kk) * ldb] : B[(k0 + kk) + (long long)gj * ldb];
        rb[q][u] = v;
      }
    }
    s_alpha = T.ar;
    s_flags = T.flags;
    s_kt = kt;
  };

  auto store = [&](int buf) {
    const uint32_t pa = sbase + buf * C::BUF, pb = pa + 2 * C::PA;
    const bool ta = s_flags & TF_TA, tb = s_flags & TF_TB;
#pragma unroll
    for (int q = 0; q < C::APER; ++q) {
      int row, kg;
      chunk_pos<BM>(ta, q, row, kg);
      uint32_t h[4], l[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) split_hl(ra[q][u] * s_alpha, h[u], l[u]);
      const uint32_t off = (uint32_t)(kg * BM + row) * 16u;
      st_shared_v4(pa + off, h[0], h[1], h[2], h[3]);
      st_shared_v4(pa + C::PA + off, l[0], l[1], l[2], l[3]);
    }
#pragma unroll
    for (int q = 0; q < C::BPER; ++q) {
      int row, kg;
      chunk_pos<BN>(!tb, q, row, kg);
      uint32_t h[4], l[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) split_hl(rb[q][u], h[u], l[u]);
      const uint32_t off = (uint32_t)(kg * BN + row) * 16u;
      st_shared_v4(pb + off, h[0], h[1], h[2], h[3]);
      st_shared_v4(pb + C::PB + off, l[0], l[1], l[2], l[3]);
    }
  };

  constexpr uint32_t idesc = tf32_idesc(BM, BN);
  UWalk w{J.t0 + it.t0, it.k0, it.kcount};
  int tt, kk, kt;
  bool have = w.next(terms, tt, kk, kt);
  if (have) load(tt, kk, kt);
  int issued = 0;        // slabs whose MMAs were committed
  bool failed = false;
  for (int c = 0; have; ++c) {
    const int buf = c & 1;
    if (c >= 2 && !mbar_wait(buf ? bar1 : bar0, ((c - 2) >> 1) & 1)) {
      abort_sh = 1;
      atomicExch(&g_umma_status, 1);
    }
    store(buf);
    const int ktc = s_kt;
    have = w.next(terms, tt, kk, kt);
    if (have) load(tt, kk, kt);
    fence_proxy_async();
    __syncthreads();
    if (abort_sh) { failed = true; break; }
    if (tid == 0) {
      fence_after();
      const uint32_t pa = sbase + buf * C::BUF, pb = pa + 2 * C::PA;
      const int nks = (ktc + 7) / 8;
      for (int s = 0; s < nks; ++s) {
        const uint32_t ao = (uint32_t)s * 2u * BM * 16u, bo = (uint32_t)s * 2u * BN * 16u;
        const uint64_t ah = kmajor_desc(pa + ao, BM * 16, 128), al = kmajor_desc(pa + C::PA + ao, BM * 16, 128);
        const uint64_t bh = kmajor_desc(pb + bo, BN * 16, 128), bl = kmajor_desc(pb + C::PB + bo, BN * 16, 128);
        umma_tf32(tmem, al, bh, idesc, (c > 0 || s > 0) ? 1u : 0u);
        umma_tf32(tmem, ah, bl, idesc, 1u);
        umma_tf32(tmem, ah, bh, idesc, 1u);
      }
      umma_commit(buf ? bar1 : bar0);
    }
    ++issued;
  }
  if (issued > 0) {
    const int last = issued - 1;
    if (!mbar_wait((last & 1) ? bar1 : bar0, (last >> 1) & 1)) {
      failed = true;
      atomicExch(&g_umma_status, 2);
    }
    // the slab before the last was waited for only if a later slab reused its buffer
  }
  failed = __syncthreads_or(failed);
  fence_after();

  if (!failed) {
    const bool direct = it.slot < 0;
    double* Cp = direct ? static_cast<double*>(bases.p[J.cbuf]) + J.coff : work + (long long)it.slot * BM * BN;
    const bool accum = J.flags & JF_ACCUM;
    const int quarter = warp & 3, half = warp >> 2;
    const int r = 32 * quarter + lane;
    constexpr int CW = BN / 2;
#pragma unroll
    for (int cc = 0; cc < CW; cc += 32) {
      uint32_t v[32];
      const int cb = half * CW + cc;
      if (issued > 0) {
        tmem_ld32(tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)cb, v);
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = 0u;
      }
      if (direct) {
        if (row0 + r < J.m) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = cb + j;
            if (col0 + col < J.n) {
              const long long idx = (row0 + r) + (long long)(col0 + col) * J.ldc;
              const double x = (double)__uint_as_float(v[j]);
              Cp[idx] = accum ? Cp[idx] + x : x;
            }
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) Cp[r + (long long)(cb + j) * BM] = (double)__uint_as_float(v[j]);
      }
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(C::TCOLS) : "memory");
  }
}

}  // namespace

int umma_tile_n() { return 64; }

void launch_items_umma(const GemmTerm* terms, const GemmJob* jobs, const WorkItem* items, int nitems, const Bases& b,
                       void* work, cudaStream_t s) {
  if (nitems <= 0) return;
  constexpr int BN = 64;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(items_umma_tf32x3<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UCfg<BN>::SMEM);
    attr = true;
  }
  items_umma_tf32x3<BN><<<nitems, kUThreads, UCfg<BN>::SMEM, s>>>(terms, jobs, items, b, static_cast<double*>(work));
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
