// svd.cu -- one-sided (Hestenes) block Jacobi SVD of the psi sector blocks.
//
// Replaces the per-sector LAPACK gesvd of the reference
// (src/dense_inst.cpp:447-541, called from src/block_tensor_inst.cpp:535-557).
// Method: Hestenes one-sided Jacobi (Hestenes 1958; Demmel & Veselic 1992,
// with the parallel block ordering of Brent & Luk and the norm-sorted column
// order of de Rijk 1989).  The C = min(m,n) columns of W (A, or A^H when m < n)
// are ordered by decreasing norm at the start of every sweep and split into
// column blocks of b = 8 or 16 (chosen per call).  Every round of a sweep
// pairs the blocks by the circle method; one CTA forms the 2b x 2b Gram matrix
// of its pair on the FP64
// tensor cores (DMMA, W streamed in row chunks), runs a cyclic sweep of the
// one-sided rotations on it, and applies the accumulated 2b x 2b rotation to
// the pair's columns of W and V (DMMA again).  Sweeps repeat until a full sweep
// performs no rotation, so the result keeps the columnwise relative accuracy of
// one-sided Jacobi on small singular values, which the reference's 1e-10
// relative cut-off depends on.
#include <cuda_runtime.h>
#include <cmath>
#include <vector>

#include "common.hpp"
#include "kernels.cuh"

namespace sadmrg {

constexpr int kSvdThreads = 512;
constexpr int kSvdWarps = kSvdThreads / 32;
// columns per block (a visit takes two blocks): 8 or 16, chosen per call by run_jacobi_svd

struct SvdPair {
  int job, bi, bj, b;   // column blocks bi, bj (bj < 0: bi alone); b = block width
};

template <bool CPLX> struct SvdT;
template <> struct SvdT<false> { using T = double; };
template <> struct SvdT<true> { using T = double2; };

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// scalar helpers for T = double / double2 (complex)
__device__ __forceinline__ double cj_mul(double a, double b) { return a * b; }   // conj(a) b
__device__ __forceinline__ double2 cj_mul(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double cmul(double a, double b) { return a * b; }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double cadd(double a, double b) { return a + b; }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double cconj(double a) { return a; }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double cre(double a) { return a; }
__device__ __forceinline__ double cre(double2 a) { return a.x; }
template <class T> __device__ __forceinline__ T czero();
template <> __device__ __forceinline__ double czero<double>() { return 0.0; }
template <> __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }

// D (8 x 8) += A (8 x 4, row-major) B (4 x 8, col-major) on the FP64 tensor cores.
// Lane l holds A(l / 4, l % 4), B(l % 4, l / 4) and D(l / 4, 2 (l % 4) + i), i = 0, 1.
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

constexpr int kChunk = 128;            // rows per streamed chunk of W or V
constexpr int kInnerMax = 1;           // inner sweeps of one visit (more cut outer sweeps by less than they cost)

template <int B>                       // B: columns per block
struct SvdGeom {
  static constexpr int Nc = 2 * B;                          // columns of one visit
  static constexpr int TD = Nc / 8;                         // 8 x 8 DMMA tiles along one side of G
  static constexpr int Ld = Nc + 1;                         // row stride of G, Q and the row chunk
  static constexpr int ChunkPer = kChunk * Nc / kSvdThreads;   // chunk elements per thread
};

template <bool CPLX, int B>
constexpr size_t svd_smem_bytes() {
  return (size_t)(2 * SvdGeom<B>::Nc + kChunk) * SvdGeom<B>::Ld * (CPLX ? 16 : 8);
}

// One visit of a column-block pair (Hestenes one-sided Jacobi in Gram form):
//   1. G = Wp^H Wp for the pair's nc <= 2B columns Wp, streamed from W in row chunks;
//   2. cyclic one-sided Jacobi on G: rotation (p, q) from a = G_pp, b = G_qq,
//      g = G_pq exactly as on the columns themselves, G <- J^H G J, Q <- Q J,
//      with the rotated diagonal set to a - t|g|, b + t|g| and G_pq to 0; up to
//      kInnerMax sweeps, stopping after a sweep that rotates nothing;
//   3. Wp <- Wp Q and Vp <- Vp Q, streamed in row chunks.
// Only G, Q and one row chunk live in shared memory, so the visit width does not
// depend on the height of the block.  The rotations rotate the Gram entries of
// the columns exactly as the column updates would (a rotation that mixes a small
// column with a large one has |s| <= sqrt(a_small / a_large)), so the entries
// keep the columnwise relative accuracy of the direct method; W itself changes
// only by the orthogonal Q.  Adds the number of rotations to *rotations.  Every
// thread of the block calls it; 16 warps, warp k owns pair k of each round.
template <bool CPLX, int B>
__device__ void jacobi_pair_visit(const SvdJob& J, const SvdPair& P, void* work, void* vmat, const int* perm,
                                  double tol, unsigned char* smem_raw, int* rotations) {
  using T = typename SvdT<CPLX>::T;
  constexpr int kNc = SvdGeom<B>::Nc, kTD = SvdGeom<B>::TD, kLdG = SvdGeom<B>::Ld;
  constexpr int kChunkPer = SvdGeom<B>::ChunkPer;
  static_assert(kSvdWarps * 2 >= kNc, "one warp per column pair of a round");
  const int R = J.trans ? J.n : J.m;
  const int C = J.trans ? J.m : J.n;
  __shared__ int cols[kNc];
  __shared__ int nrot_sh, sweep_rot_sh;
  T* G = reinterpret_cast<T*>(smem_raw);   // kNc x kLdG, row-major
  T* Q = G + kNc * kLdG;
  T* Ck = Q + kNc * kLdG;                  // kChunk x kLdG: rows of W or V, row-major
  T* W = static_cast<T*>(work) + J.woff;
  T* V = static_cast<T*>(vmat) + J.voff;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  int nc = 0;
  {
    const int n0 = min(P.b, C - P.bi * P.b);
    const int n1 = P.bj >= 0 ? min(P.b, C - P.bj * P.b) : 0;
    nc = n0 + n1;
    // block position -> column through the job's current order (columns by decreasing norm)
    const int* pj = perm + J.soff;
    if (tid < n0) cols[tid] = pj[P.bi * P.b + tid];
    else if (tid < nc) cols[tid] = pj[P.bj * P.b + (tid - n0)];
    if (tid == 0) nrot_sh = 0;
  }
  __syncthreads();

  // 1. Gram matrix on the FP64 tensor cores: warp w < kTD^2 owns the 8 x 8 tile
  //    (w / kTD, w % kTD) of G = Wp^H Wp; k runs over the rows of the chunk
  //    (zero-filled past the block)
  static_assert(kNc % 8 == 0 && kTD * kTD <= kSvdWarps, "one warp per Gram tile");
  const bool gram_warp = warp < kTD * kTD;
  const int pt = warp / kTD, qt = warp % kTD;
  const int fr = lane >> 2, fk = lane & 3;
  double g0 = 0.0, g1 = 0.0, h0 = 0.0, h1 = 0.0;   // Re (and Im) of D(fr, 2 fk + i)
  // Row chunks of a column set (W or V), read into registers one chunk ahead of
  // the one in shared memory so that the global loads overlap the products.
  T pre[kChunkPer];
  auto fetch = [&](const T* M, int ld, int r0, int rows) {
#pragma unroll
    for (int u = 0; u < kChunkPer; ++u) {
      const int e = tid + u * kSvdThreads, r = e % kChunk, c = e / kChunk;
      pre[u] = (r < rows && c < nc) ? M[(r0 + r) + (long long)cols[c] * ld] : czero<T>();
    }
  };
  auto stage = [&]() {
#pragma unroll
    for (int u = 0; u < kChunkPer; ++u) {
      const int e = tid + u * kSvdThreads, r = e % kChunk, c = e / kChunk;
      Ck[r * kLdG + c] = pre[u];
    }
  };
  fetch(W, R, 0, min(kChunk, R));
  for (int r0 = 0; r0 < R; r0 += kChunk) {
    stage();
    __syncthreads();
    if (r0 + kChunk < R) fetch(W, R, r0 + kChunk, min(kChunk, R - r0 - kChunk));
#pragma unroll 4
    for (int k0 = 0; k0 < kChunk && gram_warp; k0 += 4) {
      const T x = Ck[(k0 + fk) * kLdG + pt * 8 + fr];   // A(p, r) = conj(W(r, p))
      const T y = Ck[(k0 + fk) * kLdG + qt * 8 + fr];   // B(r, q) = W(r, q)
      if constexpr (CPLX) {
        dmma(g0, g1, x.x, y.x);
        dmma(g0, g1, x.y, y.y);
        dmma(h0, h1, x.x, y.y);
        dmma(h0, h1, -x.y, y.x);
      } else {
        dmma(g0, g1, x, y);
      }
    }
    __syncthreads();
  }
  // stored from the tiles on and above the diagonal, mirrored, so that G is exactly Hermitian
  for (int i = 0; i < 2 && gram_warp; ++i) {
    const int p = pt * 8 + fr, q = qt * 8 + 2 * fk + i;
    if (p > q) continue;
    T v;
    if constexpr (CPLX) v = make_double2(i ? g1 : g0, i ? h1 : h0);
    else v = i ? g1 : g0;
    G[p * kLdG + q] = v;
    G[q * kLdG + p] = cconj(v);
  }
  for (int e = tid; e < kNc * kNc; e += kSvdThreads) {
    const int r = e / kNc, c = e % kNc;
    Q[r * kLdG + c] = czero<T>();
    if (r == c) reinterpret_cast<double*>(Q + r * kLdG + c)[0] = 1.0;
  }
  __syncthreads();

  // a pair that needs no rotation on the fresh G keeps the inner sweep from
  // rotating at all: skip the visit when no pair of it does
  {
    int need = 0;
    for (int e = tid; e < nc * nc; e += kSvdThreads) {
      const int p = e / nc, q = e % nc;
      if (p >= q) continue;
      const double ab = cre(G[p * kLdG + p]) * cre(G[q * kLdG + q]);
      const T gpq = G[p * kLdG + q];
      double g2;
      if constexpr (CPLX) g2 = gpq.x * gpq.x + gpq.y * gpq.y; else g2 = gpq * gpq;
      if (ab > 0.0 && g2 > tol * tol * ab) need = 1;
    }
    if (!__syncthreads_or(need)) return;
  }

  // 2. inner sweeps on G
  const int N = nc + (nc & 1);
  for (int isw = 0; isw < kInnerMax && N > 1; ++isw) {
    if (tid == 0) sweep_rot_sh = 0;
    __syncthreads();
    for (int rnd = 0; rnd < N - 1; ++rnd) {
      bool act = false;
      int p = 0, q = 0;
      double c = 1.0, s = 0.0, er = 1.0, ei = 0.0, tg = 0.0, a = 0.0, b = 0.0;
      if (warp < N / 2) {
        if (warp == 0) { p = N - 1; q = rnd; }
        else { p = (rnd + warp) % (N - 1); q = (rnd - warp + (N - 1)) % (N - 1); }
        if (p > q) { const int t = p; p = q; q = t; }
        if (q < nc) {
          a = cre(G[p * kLdG + p]);
          b = cre(G[q * kLdG + q]);
          const T gpq = G[p * kLdG + q];
          double gr, gi = 0.0;
          if constexpr (CPLX) { gr = gpq.x; gi = gpq.y; } else { gr = gpq; }
          const double g2 = gr * gr + gi * gi;
          // rotate when |g| > tol sqrt(ab), compared squared; the parameters keep the
          // dependent chain of square roots and divisions short (it sets the round time)
          if (a * b > 0.0 && g2 > tol * tol * (a * b)) {
            const double g = CPLX ? sqrt(g2) : fabs(gr);
            const double ig = 1.0 / g;
            // same rotation as on the columns; for |zeta| > 1e150 zeta^2 would overflow
            const double zeta = 0.5 * (b - a) * ig;
            const double t = fabs(zeta) > 1e150 ? 0.5 / zeta
                                                : copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            if (t != 0.0) {
              act = true;
              c = rsqrt(1.0 + t * t);
              s = c * t;
              er = CPLX ? gr * ig : (gr >= 0.0 ? 1.0 : -1.0);
              ei = CPLX ? gi * ig : 0.0;
              tg = t * g;
            }
          }
        }
      }
      __syncwarp();
      // columns p, q of G and Q: [x y] <- [x y] [[c, s e^{i phi}], [-s e^{-i phi}, c]]
      if (act && lane < nc) {
        T* gpr = G + lane * kLdG;
        T* qr = Q + lane * kLdG;
        if constexpr (CPLX) {
          const double2 ep = make_double2(s * er, s * ei), em = make_double2(-s * er, s * ei);   // s e^{i phi}, -s e^{-i phi}
          double2 x = gpr[p], y = gpr[q];
          gpr[p] = cadd(make_double2(c * x.x, c * x.y), cmul(y, em));
          gpr[q] = cadd(cmul(x, ep), make_double2(c * y.x, c * y.y));
          x = qr[p]; y = qr[q];
          qr[p] = cadd(make_double2(c * x.x, c * x.y), cmul(y, em));
          qr[q] = cadd(cmul(x, ep), make_double2(c * y.x, c * y.y));
        } else {
          const double sg = s * er;
          double x = gpr[p], y = gpr[q];
          gpr[p] = c * x - sg * y;
          gpr[q] = sg * x + c * y;
          x = qr[p]; y = qr[q];
          qr[p] = c * x - sg * y;
          qr[q] = sg * x + c * y;
        }
      }
      __syncthreads();
      // rows p, q of G: G <- J^H G; the rotated 2 x 2 block is set to its exact values
      if (act && lane < nc) {
        T* rp = G + p * kLdG;
        T* rq = G + q * kLdG;
        if constexpr (CPLX) {
          const double2 x = rp[lane], y = rq[lane];
          const double2 mp = make_double2(-s * er, -s * ei), pm = make_double2(s * er, -s * ei);   // -s e^{i phi}, s e^{-i phi}
          rp[lane] = cadd(make_double2(c * x.x, c * x.y), cmul(mp, y));
          rq[lane] = cadd(cmul(pm, x), make_double2(c * y.x, c * y.y));
        } else {
          const double sg = s * er;
          const double x = rp[lane], y = rq[lane];
          rp[lane] = c * x - sg * y;
          rq[lane] = sg * x + c * y;
        }
        if (lane == p) { rp[p] = czero<T>(); reinterpret_cast<double*>(rp + p)[0] = a - tg; }
        if (lane == q) { rq[q] = czero<T>(); reinterpret_cast<double*>(rq + q)[0] = b + tg; }
        if (lane == q) rp[q] = czero<T>();
        if (lane == p) rq[p] = czero<T>();
        if (lane == 0) atomicAdd(&sweep_rot_sh, 1);
      }
      __syncthreads();
    }
    const int sr = sweep_rot_sh;
    if (tid == 0) nrot_sh += sr;
    __syncthreads();
    if (sr == 0) break;
  }
  const int nrot = nrot_sh;
  if (nrot == 0) return;        // nothing moved: W and V stay as they are

  // 3. W_pair <- W_pair Q and V_pair <- V_pair Q, in row chunks (W's, then V's): each
  //    chunk (128 x 32, zero-filled) times Q on the FP64 tensor cores (warp w: output
  //    tiles w, w + 16, ... of the 16 x 4 tile grid), the product written back over the
  //    chunk and stored coalesced; the next chunk is read while this one is multiplied
  const int nw_chunks = (R + kChunk - 1) / kChunk, nv_chunks = (C + kChunk - 1) / kChunk;
  auto chunk_of = [&](int k, T*& M, int& ld, int& r0, int& rows) {
    if (k < nw_chunks) { M = W; ld = R; r0 = k * kChunk; }
    else { M = V; ld = C; r0 = (k - nw_chunks) * kChunk; }
    rows = min(kChunk, ld - r0);
  };
  {
    T* M; int ld, r0, rows;
    chunk_of(0, M, ld, r0, rows);
    fetch(M, ld, r0, rows);
  }
  for (int k = 0; k < nw_chunks + nv_chunks; ++k) {
    T* M; int ld, r0, rows;
    chunk_of(k, M, ld, r0, rows);
    stage();
    __syncthreads();
    if (k + 1 < nw_chunks + nv_chunks) {
      T* M2; int ld2, r2, rows2;
      chunk_of(k + 1, M2, ld2, r2, rows2);
      fetch(M2, ld2, r2, rows2);
    }
    constexpr int kTiles = (kChunk / 8) * (kNc / 8) / kSvdWarps;   // output tiles per warp
    double d[kTiles][4];
#pragma unroll
    for (int u = 0; u < kTiles; ++u) {
      const int t = warp + kSvdWarps * u, rt = t / kTD, jt = t % kTD;
      double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
#pragma unroll
      for (int k0 = 0; k0 < kNc; k0 += 4) {
        const T x = Ck[(rt * 8 + fr) * kLdG + k0 + fk];
        const T y = Q[(k0 + fk) * kLdG + jt * 8 + fr];
        if constexpr (CPLX) {
          dmma(a0, a1, x.x, y.x);
          dmma(a0, a1, -x.y, y.y);
          dmma(b0, b1, x.x, y.y);
          dmma(b0, b1, x.y, y.x);
        } else {
          dmma(a0, a1, x, y);
        }
      }
      d[u][0] = a0; d[u][1] = a1; d[u][2] = b0; d[u][3] = b1;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kTiles; ++u) {
      const int t = warp + kSvdWarps * u, rt = t / kTD, jt = t % kTD;
      for (int i = 0; i < 2; ++i) {
        T v;
        if constexpr (CPLX) v = make_double2(d[u][i], d[u][2 + i]);
        else v = d[u][i];
        Ck[(rt * 8 + fr) * kLdG + jt * 8 + 2 * fk + i] = v;
      }
    }
    __syncthreads();
    for (int e = tid; e < kChunk * kNc; e += kSvdThreads) {
      const int r = e % kChunk, j = e / kChunk;
      if (r < rows && j < nc) M[(r0 + r) + (long long)cols[j] * ld] = Ck[r * kLdG + j];
    }
    __syncthreads();
  }
  if (tid == 0) atomicAdd(rotations, nrot);
}

template <bool CPLX, int B>
__global__ void __launch_bounds__(kSvdThreads) jacobi_pair_kernel(const SvdJob* __restrict__ jobs,
                                                                  const SvdPair* __restrict__ pairs, void* work,
                                                                  void* vmat, const int* perm, double tol,
                                                                  int* rotations) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SvdPair P = pairs[blockIdx.x];
  const SvdJob J = jobs[P.job];
  jacobi_pair_visit<CPLX, B>(J, P, work, vmat, perm, tol, smem_raw, rotations);
}

// ---------------------------------------------------------------------------
// All sweeps in one cooperative launch.  Rounds are separated by a grid barrier
// (bounded); rotations are counted per sector in three rotating counter sets
// (sweep s adds into set s % 3, the set of sweep s + 1 is cleared during sweep
// s, when nobody reads it any more), and a sector whose sweep made no rotation
// is skipped from then on.  Every block takes the same decisions from the same
// counts, read after the barrier that ends the sweep.
constexpr int kSvdMaxJobsCoop = 256;
constexpr unsigned long long kSvdBarrierNs = 2000000000ull;

struct SvdCtl {
  unsigned count, gen;
  int status;                 // 0, or 1 when a grid barrier ran out of time
  int sweeps;                 // sweeps taken, -1 when max_sweeps was reached
  unsigned long long t0, t1;  // device clock (ns) at the start and end of block 0
};

__device__ __forceinline__ unsigned long long svd_gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ bool svd_grid_sync(SvdCtl* ctl) {
  __shared__ int ok_sh;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok_sh = 1;
    volatile unsigned* gen = &ctl->gen;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(&ctl->count, 1u) == gridDim.x - 1) {
      atomicExch(&ctl->count, 0u);
      __threadfence();
      atomicAdd(&ctl->gen, 1u);
    } else {
      const unsigned long long t0 = svd_gtime();
      for (long long it = 0; *gen == g; ++it) {
        if (it > (1ll << 30) || ((it & 255) == 255 && svd_gtime() - t0 > kSvdBarrierNs)) {
          ok_sh = 0;
          atomicExch(&ctl->status, 1);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok_sh != 0;
}

template <bool CPLX, int B>
__global__ void __launch_bounds__(kSvdThreads) jacobi_coop_kernel(const SvdJob* __restrict__ jobs, int nj,
                                                                  const SvdPair* __restrict__ pairs,
                                                                  const int* __restrict__ roff, int max_rounds,
                                                                  void* work, void* vmat, double* nrm, int* perm,
                                                                  double tol, int* cnt, SvdCtl* ctl, int max_sweeps) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned char done[kSvdMaxJobsCoop];
  __shared__ int all_done;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->t0 = svd_gtime();
  for (int j = threadIdx.x; j < nj; j += blockDim.x) done[j] = 0;
  __syncthreads();
  int sweeps = -1;
  for (int sw = 0; sw < max_sweeps; ++sw) {
    int* cur = cnt + (sw % 3) * nj;
    if (blockIdx.x == 0)
      for (int j = threadIdx.x; j < nj; j += blockDim.x) cnt[((sw + 1) % 3) * nj + j] = 0;
    // column order of this sweep: decreasing norm (de Rijk), ties by index.  Norms
    // one warp per column, then every column's rank counted over its sector.
    {
      using T = typename SvdT<CPLX>::T;
      const int lane = threadIdx.x & 31;
      const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
      for (int j = 0; j < nj; ++j) {
        if (done[j]) continue;
        const SvdJob J = jobs[j];
        const int R = J.trans ? J.n : J.m, C = J.trans ? J.m : J.n;
        const T* W = static_cast<const T*>(work) + J.woff;
        for (int c = gw; c < C; c += nw) {
          double a = 0.0;
          for (int r = lane; r < R; r += 32) {
            const T x = W[r + (long long)c * R];
            if constexpr (CPLX) a += x.x * x.x + x.y * x.y;
            else a += x * x;
          }
          a = wsum(a);
          if (lane == 0) nrm[J.soff + c] = a;
        }
      }
      if (!svd_grid_sync(ctl)) return;
      const int gt = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
      for (int j = 0; j < nj; ++j) {
        if (done[j]) continue;
        const SvdJob J = jobs[j];
        const int C = J.trans ? J.m : J.n;
        const double* nj_ = nrm + J.soff;
        for (int c = gt; c < C; c += nt) {
          const double v = nj_[c];
          int rank = 0;
          for (int k = 0; k < C; ++k) {
            const double u = nj_[k];
            rank += (u > v || (u == v && k < c)) ? 1 : 0;
          }
          perm[J.soff + rank] = c;
        }
      }
      if (!svd_grid_sync(ctl)) return;
    }
    for (int r = 0; r < max_rounds; ++r) {
      for (int p = roff[r] + blockIdx.x; p < roff[r + 1]; p += gridDim.x) {
        const SvdPair P = pairs[p];
        if (done[P.job]) continue;
        const SvdJob J = jobs[P.job];
        jacobi_pair_visit<CPLX, B>(J, P, work, vmat, perm, tol, smem_raw, cur + P.job);
      }
      if (!svd_grid_sync(ctl)) return;
    }
    if (threadIdx.x == 0) all_done = 1;
    __syncthreads();
    for (int j = threadIdx.x; j < nj; j += blockDim.x) {
      if (!done[j] && *((volatile int*)(cur + j)) == 0) done[j] = 1;
      if (!done[j]) all_done = 0;
    }
    __syncthreads();
    if (all_done) { sweeps = sw + 1; break; }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->sweeps = sweeps;
    ctl->t1 = svd_gtime();
  }
}

// W = A (m >= n) or A^H (m < n); V = I
template <bool CPLX>
__global__ void jacobi_init_kernel(const SvdJob* jobs, const void* a, void* work, void* vmat, int* perm) {
  using T = typename SvdT<CPLX>::T;
  const SvdJob J = jobs[blockIdx.x];
  const int R = J.trans ? J.n : J.m, C = J.trans ? J.m : J.n;
  const T* A = static_cast<const T*>(a) + J.aoff;
  T* W = static_cast<T*>(work) + J.woff;
  T* V = static_cast<T*>(vmat) + J.voff;
  if (blockIdx.y == 0)
    for (int c = threadIdx.x; c < C; c += blockDim.x) perm[J.soff + c] = c;
  for (long long e = threadIdx.x + (long long)blockIdx.y * blockDim.x; e < (long long)R * C;
       e += (long long)blockDim.x * gridDim.y) {
    const int r = (int)(e % R), c = (int)(e / R);
    if (!J.trans) W[e] = A[r + (long long)c * J.m];
    else {
      T v = A[c + (long long)r * J.m];  // A^H(r, c) = conj(A(c, r))
      if (CPLX) reinterpret_cast<double2&>(v).y = -reinterpret_cast<double2&>(v).y;
      W[e] = v;
    }
  }
  for (long long e = threadIdx.x + (long long)blockIdx.y * blockDim.x; e < (long long)C * C;
       e += (long long)blockDim.x * gridDim.y) {
    const int r = (int)(e % C), c = (int)(e / C);
    if (CPLX) reinterpret_cast<double2*>(V)[e] = make_double2(r == c ? 1.0 : 0.0, 0.0);
    else reinterpret_cast<double*>(V)[e] = r == c ? 1.0 : 0.0;
  }
}

template <bool CPLX>
__global__ void jacobi_norms_kernel(const SvdJob* jobs, const void* work, double* sv) {
  using T = typename SvdT<CPLX>::T;
  const SvdJob J = jobs[blockIdx.x];
  const int R = J.trans ? J.n : J.m, C = J.trans ? J.m : J.n;
  const T* W = static_cast<const T*>(work) + J.woff;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = warp; c < C; c += nw) {
    double s = 0.0;
    for (int r = lane; r < R; r += 32) {
      if (CPLX) { const double2 v = reinterpret_cast<const double2*>(W)[r + (long long)c * R]; s += v.x * v.x + v.y * v.y; }
      else { const double v = reinterpret_cast<const double*>(W)[r + (long long)c * R]; s += v * v; }
    }
    s = wsum(s);
    if (lane == 0) sv[J.soff + c] = sqrt(s);
  }
}

// Host driver.  Runs all sweeps in one cooperative launch when the device allows
// it, otherwise one launch per round and one host synchronisation per sweep to
// test convergence.  Returns the number of sweeps taken (or -1 when max_sweeps
// was reached).
template <bool CPLX, int B>
static int jacobi_run(const void* a, void* work, void* vmat, double* sv, const std::vector<SvdJob>& hjobs,
                      int max_sweeps, cudaStream_t s, double* kernel_ms) {
  const int nj = (int)hjobs.size();
  std::vector<int> bsz(nj), nblk(nj), nrounds(nj);
  int max_rounds = 0, maxR = 0;
  size_t smem = 0;
  for (int j = 0; j < nj; ++j) {
    const int R = hjobs[j].trans ? hjobs[j].n : hjobs[j].m;
    const int C = hjobs[j].trans ? hjobs[j].m : hjobs[j].n;
    maxR = std::max(maxR, R);
    bsz[j] = B;
    nblk[j] = (C + bsz[j] - 1) / bsz[j];
    const int N = nblk[j] + (nblk[j] & 1);
    nrounds[j] = nblk[j] <= 1 ? 1 : N - 1;
    max_rounds = std::max(max_rounds, nrounds[j]);
    smem = svd_smem_bytes<CPLX, B>();
  }
  // pair lists per round
  std::vector<std::vector<SvdPair>> rounds(max_rounds);
  for (int j = 0; j < nj; ++j) {
    if (nblk[j] <= 1) { rounds[0].push_back({j, 0, -1, bsz[j]}); continue; }
    const int N = nblk[j] + (nblk[j] & 1);
    for (int r = 0; r < N - 1; ++r)
      for (int i = 0; i < N / 2; ++i) {
        int p, q;
        if (i == 0) { p = N - 1; q = r; }
        else { p = (r + i) % (N - 1); q = (r - i + (N - 1)) % (N - 1); }
        if (p >= nblk[j] || q >= nblk[j]) continue;
        rounds[r].push_back({j, std::min(p, q), std::max(p, q), bsz[j]});
      }
  }
  std::vector<int> roff(max_rounds + 1, 0);
  std::vector<SvdPair> flat;
  for (int r = 0; r < max_rounds; ++r) {
    roff[r] = (int)flat.size();
    flat.insert(flat.end(), rounds[r].begin(), rounds[r].end());
  }
  roff[max_rounds] = (int)flat.size();
  long long nsv = 1;   // singular-value slots (the column order lives at the same offsets)
  for (int j = 0; j < nj; ++j)
    nsv = std::max<long long>(nsv, hjobs[j].soff + (hjobs[j].trans ? hjobs[j].m : hjobs[j].n));
  DevBuf djobs(sizeof(SvdJob) * nj, s), dpairs(sizeof(SvdPair) * flat.size(), s), dcnt(sizeof(int), s),
      dperm(sizeof(int) * nsv, s);
  SADMRG_CUDA(cudaMemcpyAsync(djobs.get(), hjobs.data(), sizeof(SvdJob) * nj, cudaMemcpyHostToDevice, s));
  SADMRG_CUDA(cudaMemcpyAsync(dpairs.get(), flat.data(), sizeof(SvdPair) * flat.size(), cudaMemcpyHostToDevice, s));
  dim3 ig(nj, 16);
  jacobi_init_kernel<CPLX><<<ig, 256, 0, s>>>(djobs.as<SvdJob>(), a, work, vmat, dperm.as<int>());
  SADMRG_CUDA(cudaGetLastError());
  SADMRG_CUDA(cudaFuncSetAttribute(jacobi_pair_kernel<CPLX, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const double tol = std::sqrt((double)std::max(maxR, 1)) * 2.220446049250313e-16;
  int sweeps = -1;
  int h_rot = 0;
  // preferred: every sweep in one cooperative launch (no host round trip per sweep)
  int dev = 0, coop = 0, nsm = 0, per_sm = 0;
  SADMRG_CUDA(cudaGetDevice(&dev));
  SADMRG_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  SADMRG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  SADMRG_CUDA(cudaFuncSetAttribute(jacobi_coop_kernel<CPLX, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  SADMRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_coop_kernel<CPLX, B>, kSvdThreads, smem));
  int max_pairs = 1;
  for (int r = 0; r < max_rounds; ++r) max_pairs = std::max(max_pairs, roff[r + 1] - roff[r]);
  if (coop && per_sm > 0 && nj <= kSvdMaxJobsCoop) {
    const int grid = std::max(1, std::min(max_pairs, per_sm * nsm));
    DevBuf droff(sizeof(int) * (max_rounds + 1), s), dcnt3(sizeof(int) * 3 * nj, s), dctl(sizeof(SvdCtl), s);
    SADMRG_CUDA(cudaMemcpyAsync(droff.get(), roff.data(), sizeof(int) * (max_rounds + 1), cudaMemcpyHostToDevice, s));
    SADMRG_CUDA(cudaMemsetAsync(dcnt3.get(), 0, sizeof(int) * 3 * nj, s));
    SADMRG_CUDA(cudaMemsetAsync(dctl.get(), 0, sizeof(SvdCtl), s));
    const SvdJob* pj = djobs.as<SvdJob>();
    const SvdPair* pp = dpairs.as<SvdPair>();
    const int* pr = droff.as<int>();
    int* pc = dcnt3.as<int>();
    SvdCtl* pctl = dctl.as<SvdCtl>();
    int njv = nj, mr = max_rounds, ms = max_sweeps;
    double tolv = tol;
    void* a_work = work;
    void* a_vmat = vmat;
    double* a_nrm = sv;   // column norms of each sweep; the final singular values overwrite them
    int* a_perm = dperm.as<int>();
    void* args[] = {(void*)&pj,     (void*)&njv,    (void*)&pp,   (void*)&pr, (void*)&mr,   (void*)&a_work,
                    (void*)&a_vmat, (void*)&a_nrm, (void*)&a_perm, (void*)&tolv, (void*)&pc, (void*)&pctl,
                    (void*)&ms};
    SADMRG_CUDA(cudaLaunchCooperativeKernel((const void*)jacobi_coop_kernel<CPLX, B>, dim3(grid), dim3(kSvdThreads),
                                            args, smem, s));
    SvdCtl hctl{};
    SADMRG_CUDA(cudaMemcpyAsync(&hctl, dctl.get(), sizeof(SvdCtl), cudaMemcpyDeviceToHost, s));
    SADMRG_CUDA(cudaStreamSynchronize(s));
    SADMRG_REQUIRE(hctl.status == 0, SADMRG_ERR_CUDA, "jacobi svd: a grid barrier ran out of time");
    sweeps = hctl.sweeps;
    if (kernel_ms) *kernel_ms = (double)(hctl.t1 - hctl.t0) * 1e-6;
    jacobi_norms_kernel<CPLX><<<nj, 256, 0, s>>>(djobs.as<SvdJob>(), work, sv);
    SADMRG_CUDA(cudaGetLastError());
    return sweeps;
  }
  for (int sw = 0; sw < max_sweeps; ++sw) {
    SADMRG_CUDA(cudaMemsetAsync(dcnt.get(), 0, sizeof(int), s));
    for (int r = 0; r < max_rounds; ++r) {
      const int np = roff[r + 1] - roff[r];
      if (np == 0) continue;
      jacobi_pair_kernel<CPLX, B><<<np, kSvdThreads, smem, s>>>(djobs.as<SvdJob>(), dpairs.as<SvdPair>() + roff[r],
                                                                work, vmat, dperm.as<int>(), tol, dcnt.as<int>());
    }
    SADMRG_CUDA(cudaGetLastError());
    SADMRG_CUDA(cudaMemcpyAsync(&h_rot, dcnt.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    SADMRG_CUDA(cudaStreamSynchronize(s));
    if (h_rot == 0) { sweeps = sw + 1; break; }
  }
  jacobi_norms_kernel<CPLX><<<nj, 256, 0, s>>>(djobs.as<SvdJob>(), work, sv);
  SADMRG_CUDA(cudaGetLastError());
  return sweeps;
}

int run_jacobi_svd(bool cplx, const void* a, void* work, void* vmat, double* sv, const std::vector<SvdJob>& hjobs,
                   int max_sweeps, cudaStream_t s, double* kernel_ms) {
  if (kernel_ms) *kernel_ms = -1.0;
  if (hjobs.empty()) return 0;
  // column blocks of 16, or of 8 when the widest round of 16-column pairs would
  // keep fewer than half the SMs busy: narrower pairs double the CTAs per round
  // and cut each visit's work to a quarter, which wins while SMs are idle (D=512:
  // 1.87 -> 1.65 s of SVD per sweep) and loses once they are not (complex D=2048:
  // 4.8 -> 5.5 s per iDMRG)
  int dev = 0, nsm = 0;
  SADMRG_CUDA(cudaGetDevice(&dev));
  SADMRG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  long long pairs16 = 0;
  for (const SvdJob& J : hjobs) {
    const int C = J.trans ? J.m : J.n;
    const int nb = (C + 15) / 16;
    pairs16 += nb <= 1 ? 1 : nb / 2;
  }
  const bool narrow = 2 * pairs16 < nsm;
  if (cplx)
    return narrow ? jacobi_run<true, 8>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms)
                  : jacobi_run<true, 16>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms);
  return narrow ? jacobi_run<false, 8>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms)
                : jacobi_run<false, 16>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms);
}

}  // namespace sadmrg
