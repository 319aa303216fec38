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
#include <algorithm>
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

// 2^-k for a normal double m = 2^k (1 + f): m times it lies in [1, 2) (built from the
// exponent bits, exact)
__device__ __forceinline__ double pow2_scale_of(double m) {
  const int e = (__double2hiint(m) >> 20) & 0x7ff;
  return __hiloint2double((2046 - e) << 20, 0);
}
// The one-sided rotation of a pair with squared norms a, b and |<w_p, w_q>| = g > 0,
// as on the columns themselves: t = tan(theta) = 2 g sgn(d) / (|d| + r) with d = b - a,
// r = sqrt(d^2 + 4 g^2).  With u = |d| + r and q = 1 / sqrt(2 r u) (since
// 1 + t^2 = 2 r / u): c = cos(theta) = u q, s = sin(theta) = 2 g q sgn(d) and
// t = 4 g r q^2 sgn(d) -- two inverse square roots and no division on the chain
// that sets the time of an inner round.  d and g are first scaled by a power of two
// (the larger of |d| and 2 g into [1, 2)), so that the squares neither overflow nor
// underflow; c, s and t do not depend on the scale.  Returns c, s and t g.
__device__ __forceinline__ void jacobi_rotation(double a, double b, double g, double& c, double& s, double& tg) {
  const double d = b - a;
  const double sc = pow2_scale_of(fmax(fabs(d), 2.0 * g));
  const double dn = d * sc, gn = g * sc;
  const double x = fma(dn, dn, 4.0 * gn * gn);
  const double r = x * rsqrt(x);
  const double u = fabs(dn) + r;
  const double q = rsqrt(2.0 * r * u);
  const double sg = d >= 0.0 ? 1.0 : -1.0;
  c = u * q;
  s = sg * (2.0 * gn * q);
  tg = sg * (4.0 * gn * r * q * q) * g;
}

// One element (8 or 16 bytes) copied global -> shared without passing through
// registers (cp.async, Ampere and later); zero-filled instead when !ok (src must
// still be a valid address).
template <class T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src, bool ok) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(src), "r"(ok ? 16 : 0) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(src), "r"(ok ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// all but the most recently committed group of this thread's copies have landed
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

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
constexpr size_t svd_smem_bytes() {   // G, Q and two row-chunk buffers
  return (size_t)(2 * SvdGeom<B>::Nc + 2 * kChunk) * SvdGeom<B>::Ld * (CPLX ? 16 : 8);
}
// shared memory of a resident visit (all rows of the pair's W and V columns) of a
// block with R + C rows in total; launches whose largest pair needs more stream
// row chunks instead
template <bool CPLX, int B>
constexpr size_t svd_res_smem_bytes(long long rows) {
  return (size_t)(2 * SvdGeom<B>::Nc + rows) * SvdGeom<B>::Ld * (CPLX ? 16 : 8) + (size_t)kSvdWarps * 32 * 4 * 8;
}
constexpr size_t kSvdResMax = 160 * 1024;

// One visit of a column-block pair (Hestenes one-sided Jacobi in Gram form):
//   1. G = Wp^H Wp for the pair's nc <= 2B columns Wp, streamed from W in row chunks;
//   2. cyclic one-sided Jacobi on G: rotation (p, q) from a = G_pp, b = G_qq,
//      g = G_pq exactly as on the columns themselves, G <- J^H G J, Q <- Q J,
//      with the rotated diagonal set to a - t|g|, b + t|g| and G_pq to 0; up to
//      kInnerMax sweeps, stopping after a sweep that rotates nothing;
//   3. Wp <- Wp Q and Vp <- Vp Q, streamed in row chunks.
// Only G, Q and one row chunk live in shared memory, so the visit width does not
// depend on the height of the block -- or, when the launch's largest pair fits
// (res), all rows of the pair's columns of W and V: one load, the Gram tiles with
// their rows split over all warps (partials summed in a fixed order), and Q applied
// in place by warps that own whole 8-row tiles.  The rotations rotate the Gram entries of
// the columns exactly as the column updates would (a rotation that mixes a small
// column with a large one has |s| <= sqrt(a_small / a_large)), so the entries
// keep the columnwise relative accuracy of the direct method; W itself changes
// only by the orthogonal Q.  Adds the number of rotations to *rotations.  Every
// thread of the block calls it; 16 warps, warp k owns pair k of each round.
template <bool CPLX, int B>
__device__ void jacobi_pair_visit(const SvdJob& J, const SvdPair& P, void* work, void* vmat, const int* perm,
                                  double tol, unsigned char* smem_raw, int* rotations, bool res) {
  using T = typename SvdT<CPLX>::T;
  constexpr int kNc = SvdGeom<B>::Nc, kTD = SvdGeom<B>::TD, kLdG = SvdGeom<B>::Ld;
  constexpr int kChunkPer = SvdGeom<B>::ChunkPer;
  static_assert(kSvdWarps * 2 >= kNc, "one warp per column pair of a round");
  const int R = J.trans ? J.n : J.m;
  const int C = J.trans ? J.m : J.n;
  __shared__ int cols[kNc];
  T* G = reinterpret_cast<T*>(smem_raw);   // kNc x kLdG, row-major
  T* Q = G + kNc * kLdG;
  T* Ck = Q + kNc * kLdG;                  // kChunk x kLdG: rows of W or V, row-major
  // resident visit: all R rows of the pair's W columns, then all C rows of its V columns
  T* Ws = Ck;
  T* Vs = Ws + R * kLdG;
  double* Gp = reinterpret_cast<double*>(Vs + C * kLdG);   // Gram partials, 4 per lane per warp
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
  }
  __syncthreads();

  // 1. Gram matrix on the FP64 tensor cores: warp w < kTD^2 owns the 8 x 8 tile
  //    (w / kTD, w % kTD) of G = Wp^H Wp; k runs over the rows of the chunk
  //    (zero-filled past the block)
  static_assert(kNc % 8 == 0 && kTD * kTD <= kSvdWarps, "one warp per Gram tile");
  constexpr int kTiles = kTD * kTD, kSplit = kSvdWarps / kTiles;
  const bool gram_warp = warp < kTiles;
  const int fr = lane >> 2, fk = lane & 3;
  double g0 = 0.0, g1 = 0.0, h0 = 0.0, h1 = 0.0;   // Re (and Im) of D(fr, 2 fk + i)
  // Streamed visits: row chunks of a column set (W or V) copied asynchronously
  // into two shared buffers, the next chunk in flight while one is multiplied
  // (rows past the block and columns past nc zero-filled); one group per chunk.
  T* const Cb0 = Ck;
  T* const Cb1 = Ck + kChunk * kLdG;
  auto issue = [&](const T* M, int ld, int r0, int rows, T* dst) {
#pragma unroll
    for (int u = 0; u < kChunkPer; ++u) {
      const int e = tid + u * kSvdThreads, r = e % kChunk, c = e / kChunk;
      const bool ok = r < rows && c < nc;
      cp_async_elem(dst + r * kLdG + c, ok ? M + (r0 + r) + (long long)cols[c] * ld : M, ok);
    }
    cp_async_commit();
  };
  if (res) {
    // one load of everything the visit touches (columns past nc zero-filled), then
    // the Gram tiles with their rows split over all warps: warp w computes tile
    // w % kTiles over the w / kTiles-th part of the rows; the parts are summed in
    // part order
    // one thread per row of W then V, its columns read into registers together so
    // that all of a thread's loads are in flight at once (coalesced along rows)
    constexpr int kU = CPLX ? 8 : 16;
    for (int r0 = 0; r0 < R + C; r0 += kSvdThreads) {
      const int rr = r0 + tid;
      if (rr < R + C) {
        const bool isw = rr < R;
        const int r = isw ? rr : rr - R, ld = isw ? R : C;
        const T* M = isw ? W : V;
        T* D = (isw ? Ws : Vs) + r * kLdG;
#pragma unroll
        for (int c0 = 0; c0 < kNc; c0 += kU) {
          T v[kU];
#pragma unroll
          for (int u = 0; u < kU; ++u) v[u] = c0 + u < nc ? M[r + (long long)cols[c0 + u] * ld] : czero<T>();
#pragma unroll
          for (int u = 0; u < kU; ++u) D[c0 + u] = v[u];
        }
      }
    }
    __syncthreads();
    const int tile = warp % kTiles, part = warp / kTiles;
    const int pt = tile / kTD, qt = tile % kTD;
    const int rs = (((R + kSplit - 1) / kSplit) + 3) & ~3;
    const int k0s = part * rs, k1s = min(R, k0s + rs);
    for (int k0 = k0s; k0 < k1s; k0 += 4) {
      const int k = k0 + fk;
      const T x = k < k1s ? Ws[k * kLdG + pt * 8 + fr] : czero<T>();   // A(p, r) = conj(W(r, p))
      const T y = k < k1s ? Ws[k * kLdG + qt * 8 + fr] : czero<T>();   // B(r, q) = W(r, q)
      if constexpr (CPLX) {
        dmma(g0, g1, x.x, y.x);
        dmma(g0, g1, x.y, y.y);
        dmma(h0, h1, x.x, y.y);
        dmma(h0, h1, -x.y, y.x);
      } else {
        dmma(g0, g1, x, y);
      }
    }
    if constexpr (kSplit > 1) {
      if (part > 0) {
        double* o = Gp + (warp * 32 + lane) * 4;
        o[0] = g0; o[1] = g1; o[2] = h0; o[3] = h1;
      }
      __syncthreads();
      if (part == 0)
        for (int pp = 1; pp < kSplit; ++pp) {
          const double* o = Gp + ((tile + pp * kTiles) * 32 + lane) * 4;
          g0 += o[0]; g1 += o[1]; h0 += o[2]; h1 += o[3];
        }
    }
  } else {
    const int pt = warp / kTD, qt = warp % kTD;
    const int nch = (R + kChunk - 1) / kChunk;
    issue(W, R, 0, min(kChunk, R), Cb0);
    if (nch > 1) issue(W, R, kChunk, min(kChunk, R - kChunk), Cb1);
    else cp_async_commit();
    double e0 = 0.0, e1 = 0.0, f0 = 0.0, f1 = 0.0;   // a second chain over the odd k steps
    for (int ch = 0; ch < nch; ++ch) {
      cp_async_wait1();
      __syncthreads();
      const T* Cc = (ch & 1) ? Cb1 : Cb0;
      if (gram_warp) {
#pragma unroll 4
        for (int k0 = 0; k0 < kChunk; k0 += 8) {
          const T x = Cc[(k0 + fk) * kLdG + pt * 8 + fr];       // A(p, r) = conj(W(r, p))
          const T y = Cc[(k0 + fk) * kLdG + qt * 8 + fr];       // B(r, q) = W(r, q)
          const T x2 = Cc[(k0 + 4 + fk) * kLdG + pt * 8 + fr];
          const T y2 = Cc[(k0 + 4 + fk) * kLdG + qt * 8 + fr];
          if constexpr (CPLX) {
            dmma(g0, g1, x.x, y.x);
            dmma(g0, g1, x.y, y.y);
            dmma(h0, h1, x.x, y.y);
            dmma(h0, h1, -x.y, y.x);
            dmma(e0, e1, x2.x, y2.x);
            dmma(e0, e1, x2.y, y2.y);
            dmma(f0, f1, x2.x, y2.y);
            dmma(f0, f1, -x2.y, y2.x);
          } else {
            dmma(g0, g1, x, y);
            dmma(e0, e1, x2, y2);
          }
        }
      }
      __syncthreads();
      if (ch + 2 < nch) issue(W, R, (ch + 2) * kChunk, min(kChunk, R - (ch + 2) * kChunk), (ch & 1) ? Cb1 : Cb0);
      else cp_async_commit();
    }
    g0 += e0; g1 += e1; h0 += f0; h1 += f1;
  }
  // stored from the tiles on and above the diagonal, mirrored, so that G is exactly Hermitian
  const int pt = warp / kTD, qt = warp % kTD;
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
  int nrot = 0;
  for (int isw = 0; isw < kInnerMax && N > 1; ++isw) {
    int sr = 0;   // rotations of this inner sweep (the same count in every thread)
    for (int rnd = 0; rnd < N - 1; ++rnd) {
      bool act = false;
      int p = 0, q = 0;
      double c = 1.0, s = 0.0, er = 1.0, ei = 0.0, tg = 0.0, a = 0.0, b = 0.0;
      if (warp < N / 2) {
        if (warp == 0) { p = N - 1; q = rnd; }
        else {
          p = rnd + warp;
          if (p >= N - 1) p -= N - 1;
          q = rnd - warp;
          if (q < 0) q += N - 1;
        }
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
            double g;
            if constexpr (CPLX) {
              g = sqrt(g2);
              const double ig = 1.0 / g;
              er = gr * ig;
              ei = gi * ig;
            } else {
              g = fabs(gr);
              er = gr >= 0.0 ? 1.0 : -1.0;
            }
            jacobi_rotation(a, b, g, c, s, tg);
            act = true;
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
      }
      sr += __syncthreads_count(act && lane == 0);
    }
    nrot += sr;
    if (sr == 0) break;
  }
  if (nrot == 0) return;        // nothing moved: W and V stay as they are

  if (res) {
    // 3. Ws <- Ws Q and Vs <- Vs Q in place: warp w owns the 8-row tiles w, w + 16, ...
    //    of the rows of Ws then Vs and computes all their output columns before it
    //    writes them back; then every thread stores the new columns
    const int ntw = (R + 7) / 8, ntv = (C + 7) / 8;
    for (int t = warp; t < ntw + ntv; t += kSvdWarps) {
      T* M = t < ntw ? Ws : Vs;
      const int rows = t < ntw ? R : C, r = (t < ntw ? t : t - ntw) * 8 + fr;
      double acc[kTD][4];
#pragma unroll
      for (int jt = 0; jt < kTD; ++jt) acc[jt][0] = acc[jt][1] = acc[jt][2] = acc[jt][3] = 0.0;
#pragma unroll
      for (int k0 = 0; k0 < kNc; k0 += 4) {
        const T x = r < rows ? M[r * kLdG + k0 + fk] : czero<T>();
#pragma unroll
        for (int jt = 0; jt < kTD; ++jt) {
          const T y = Q[(k0 + fk) * kLdG + jt * 8 + fr];
          if constexpr (CPLX) {
            dmma(acc[jt][0], acc[jt][1], x.x, y.x);
            dmma(acc[jt][0], acc[jt][1], -x.y, y.y);
            dmma(acc[jt][2], acc[jt][3], x.x, y.y);
            dmma(acc[jt][2], acc[jt][3], x.y, y.x);
          } else {
            dmma(acc[jt][0], acc[jt][1], x, y);
          }
        }
      }
      __syncwarp();
      if (r < rows) {
#pragma unroll
        for (int jt = 0; jt < kTD; ++jt)
          for (int i = 0; i < 2; ++i) {
            T v;
            if constexpr (CPLX) v = make_double2(acc[jt][i], acc[jt][2 + i]);
            else v = acc[jt][i];
            M[r * kLdG + jt * 8 + 2 * fk + i] = v;
          }
      }
    }
    __syncthreads();
    for (int r0 = 0; r0 < R + C; r0 += kSvdThreads) {
      const int rr = r0 + tid;
      if (rr < R + C) {
        const bool isw = rr < R;
        const int r = isw ? rr : rr - R, ld = isw ? R : C;
        T* M = isw ? W : V;
        const T* S = (isw ? Ws : Vs) + r * kLdG;
#pragma unroll
        for (int c = 0; c < kNc; ++c)
          if (c < nc) M[r + (long long)cols[c] * ld] = S[c];
      }
    }
    __syncthreads();   // the next visit of this CTA reloads the shared arrays
    if (tid == 0) atomicAdd(rotations, nrot);
    return;
  }

  // 3. W_pair <- W_pair Q and V_pair <- V_pair Q, in row chunks (W's, then V's): each
  //    chunk (128 x 2B, zero-filled) times Q on the FP64 tensor cores (warp w: output
  //    tiles w, w + 16, ... of the chunk's 8 x 8 tile grid), the products stored
  //    from registers; the chunk after next is copied in while one is multiplied
  const int nw_chunks = (R + kChunk - 1) / kChunk, nv_chunks = (C + kChunk - 1) / kChunk;
  const int nall = nw_chunks + nv_chunks;
  auto chunk_of = [&](int k, T*& M, int& ld, int& r0, int& rows) {
    if (k < nw_chunks) { M = W; ld = R; r0 = k * kChunk; }
    else { M = V; ld = C; r0 = (k - nw_chunks) * kChunk; }
    rows = min(kChunk, ld - r0);
  };
  for (int k = 0; k < 2; ++k) {
    if (k < nall) {
      T* M; int ld, r0, rows;
      chunk_of(k, M, ld, r0, rows);
      issue(M, ld, r0, rows, k ? Cb1 : Cb0);
    } else {
      cp_async_commit();
    }
  }
  for (int k = 0; k < nall; ++k) {
    T* M; int ld, r0, rows;
    chunk_of(k, M, ld, r0, rows);
    cp_async_wait1();
    __syncthreads();
    const T* Cc = (k & 1) ? Cb1 : Cb0;
    constexpr int kTiles = (kChunk / 8) * (kNc / 8) / kSvdWarps;   // output tiles per warp
#pragma unroll
    for (int u = 0; u < kTiles; ++u) {
      const int t = warp + kSvdWarps * u, rt = t / kTD, jt = t % kTD;
      double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
#pragma unroll
      for (int k0 = 0; k0 < kNc; k0 += 4) {
        const T x = Cc[(rt * 8 + fr) * kLdG + k0 + fk];
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
      const int r = rt * 8 + fr;
      if (r < rows) {
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int j = jt * 8 + 2 * fk + i;
          if (j >= nc) continue;
          T v;
          if constexpr (CPLX) v = make_double2(i ? a1 : a0, i ? b1 : b0);
          else v = i ? a1 : a0;
          M[(r0 + r) + (long long)cols[j] * ld] = v;
        }
      }
    }
    __syncthreads();   // every warp is done with this buffer
    if (k + 2 < nall) {
      T* M2; int ld2, r2, rows2;
      chunk_of(k + 2, M2, ld2, r2, rows2);
      issue(M2, ld2, r2, rows2, (k & 1) ? Cb1 : Cb0);
    } else {
      cp_async_commit();
    }
  }
  if (tid == 0) atomicAdd(rotations, nrot);
}

template <bool CPLX, int B>
__global__ void __launch_bounds__(kSvdThreads) jacobi_pair_kernel(const SvdJob* __restrict__ jobs,
                                                                  const SvdPair* __restrict__ pairs, void* work,
                                                                  void* vmat, const int* perm, double tol,
                                                                  int* rotations, int res) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SvdPair P = pairs[blockIdx.x];
  const SvdJob J = jobs[P.job];
  jacobi_pair_visit<CPLX, B>(J, P, work, vmat, perm, tol, smem_raw, rotations, res != 0);
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
                                                                  double tol, int* cnt, SvdCtl* ctl, int max_sweeps,
                                                                  int res) {
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
        jacobi_pair_visit<CPLX, B>(J, P, work, vmat, perm, tol, smem_raw, cur + P.job, res != 0);
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

// W = A (m >= n) or A^H (m < n); V = I (copy = 0: only the column order, when the
// caller has set W and V itself)
template <bool CPLX>
__global__ void jacobi_init_kernel(const SvdJob* jobs, const void* a, void* work, void* vmat, int* perm, int copy) {
  using T = typename SvdT<CPLX>::T;
  const SvdJob J = jobs[blockIdx.x];
  const int R = J.trans ? J.n : J.m, C = J.trans ? J.m : J.n;
  const T* A = static_cast<const T*>(a) + J.aoff;
  T* W = static_cast<T*>(work) + J.woff;
  T* V = static_cast<T*>(vmat) + J.voff;
  if (blockIdx.y == 0)
    for (int c = threadIdx.x; c < C; c += blockDim.x) perm[J.soff + c] = c;
  if (!copy) return;
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

// ---------------------------------------------------------------------------
// QR preconditioning (Drmac & Veselic, "New fast and accurate Jacobi SVD
// algorithm I", SIAM J. Matrix Anal. Appl. 29, 2008): with the columns of
// W0 = op(A) ordered by decreasing norm (P), W0 = Q R and R^H = Q1 R1 by
// Householder reflections, and the one-sided Jacobi runs on R1^H (C x C) instead
// of W0:
//   R1^H V2 = U2 S  =>  op(A) = (Q U2) S (P Q1 V2)^H,
// so the outputs keep the meaning they have without preconditioning -- W =
// Q [R1^H V2; 0] = Q U2 S, the left factor times S, and V = P Q1 V2 -- with no
// division by S.  The graded rows of R make the Jacobi converge in well under
// the sweeps it takes on W0 itself.  Each QR is
// blocked (panels of NB columns, compact WY form H_1 ... H_NB = I - Y T Y^H as in
// LAPACK's larft): one CTA factors a job's panel in shared memory, then every
// CTA updates one NB-column tile of a trailing matrix; Q (V1 S) applies the same
// block reflectors in reverse.  All panels run in one cooperative launch with
// bounded grid barriers.
template <bool CPLX> struct QrGeom {
  static constexpr int NB = CPLX ? 8 : 16;     // panel width
  static constexpr int RC = 256;               // rows per chunk of a tile update
  static constexpr int LD = RC + 1;            // shared row stride of a chunk (odd: no bank conflicts)
  static constexpr int NT = NB * NB;
  static constexpr int G = kSvdThreads / NT;   // row groups of the Y = V^H X sums
};
constexpr size_t kQrSmemMax = 200 * 1024;       // largest panel kept in shared memory
// Calls whose widest block has fewer columns run the Jacobi directly: it needs a
// few rounds per sweep there, so the QRs would cost about what they save.  (It
// also keeps the first steps of an iDMRG warm-up -- blocks of a few columns,
// some of pure rounding noise, whose kept count the 1e-16 floor of the
// per-sector cut-off then decides -- on the path of the plain Jacobi.)
constexpr int kQrMinCols = 32;

struct QrJob {
  long long aoff;             // input block (m x n, lda m)
  long long qoff;             // the matrix factored (R x C, ld R), then R above and the reflectors below the diagonal
  long long toff;             // T factors of the panels, NB x NB each (column-major)
  long long jwoff, jvoff;     // the Jacobi's W = R1^H and V (C x C each)
  long long woff, voff, soff; // outputs as in SvdJob; for a Q application: the matrix it multiplies (ld R)
  int m, n, trans, R, C;
  int x_in_q;                 // Q application: the matrix is in the QR buffer (1) or in the output W (0)
};
struct QrTile {
  int job, c1;                // a tile of NB columns starting at column c1
};

__device__ __forceinline__ double cabs2(double a) { return a * a; }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double cim(double) { return 0.0; }
__device__ __forceinline__ double cim(double2 a) { return a.y; }
__device__ __forceinline__ double csub(double a, double b) { return a - b; }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
template <class T> __device__ __forceinline__ T cmake(double re, double im);
template <> __device__ __forceinline__ double cmake<double>(double re, double) { return re; }
template <> __device__ __forceinline__ double2 cmake<double2>(double re, double im) { return make_double2(re, im); }
__device__ __forceinline__ double wsum_t(double v) { return wsum(v); }
__device__ __forceinline__ double2 wsum_t(double2 v) { return make_double2(wsum(v.x), wsum(v.y)); }
__device__ __forceinline__ double cscale(double a, double s) { return a * s; }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// column c of op(A) at row r: A(r, c), or conj(A(c, r)) when the job works on A^H
template <class T>
__device__ __forceinline__ T op_a(const T* A, int m, int trans, int r, int c) {
  return trans ? cconj(A[c + (long long)r * m]) : A[r + (long long)c * m];
}

// Column norms of op(A) and their order (decreasing, ties by index): P.
template <bool CPLX>
__global__ void qr_order_kernel(const QrJob* jobs, const void* a, double* nrm, int* perm) {
  using T = typename SvdT<CPLX>::T;
  const QrJob J = jobs[blockIdx.x];
  const T* A = static_cast<const T*>(a) + J.aoff;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* nj = nrm + J.soff;
  for (int c = warp; c < J.C; c += nw) {
    double s = 0.0;
    for (int r = lane; r < J.R; r += 32) s += cabs2(op_a(A, J.m, J.trans, r, c));
    s = wsum(s);
    if (lane == 0) nj[c] = s;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < J.C; c += blockDim.x) {
    const double v = nj[c];
    int rank = 0;
    for (int k = 0; k < J.C; ++k) {
      const double u = nj[k];
      rank += (u > v || (u == v && k < c)) ? 1 : 0;
    }
    perm[J.soff + rank] = c;
  }
}

// W0 = op(A) P
template <bool CPLX>
__global__ void qr_gather_kernel(const QrJob* jobs, const void* a, void* qbuf, const int* perm) {
  using T = typename SvdT<CPLX>::T;
  const QrJob J = jobs[blockIdx.x];
  const T* A = static_cast<const T*>(a) + J.aoff;
  T* W = static_cast<T*>(qbuf) + J.qoff;
  const int* p = perm + J.soff;
  for (long long e = threadIdx.x + (long long)blockIdx.y * blockDim.x; e < (long long)J.R * J.C;
       e += (long long)blockDim.x * gridDim.y) {
    const int r = (int)(e % J.R), i = (int)(e / J.R);
    W[e] = op_a(A, J.m, J.trans, r, p[i]);
  }
}

// Panel k of job J: Householder reflections of its NB columns (rows k NB .. R-1)
// in shared memory (LAPACK larfg: beta = -sign(Re alpha) |x|, tau = (beta -
// alpha) / beta, v = x / (alpha - beta) below the unit diagonal; no reflection
// when the column below the diagonal is zero and alpha is real), each applied as
// H^H to the panel's later columns; then T of the compact WY form (forward,
// columnwise).  Writes R's panel rows, the reflectors and T back.
template <bool CPLX>
__device__ void qr_panel(const QrJob& J, int k, void* qbuf, unsigned char* smem) {
  using T = typename SvdT<CPLX>::T;
  constexpr int NB = QrGeom<CPLX>::NB;
  const int r0 = k * NB, nr = J.R - r0, w = min(NB, J.C - r0);
  T* A = static_cast<T*>(qbuf) + J.qoff;
  T* P = reinterpret_cast<T*>(smem);   // nr x w, column-major, ld nr
  __shared__ T tau_sh[NB];
  __shared__ T S_sh[NB * NB];          // S(k, j) = v_k^H v_j, k < j
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < nr * w; e += blockDim.x) {
    const int i = e % nr, l = e / nr;
    P[e] = A[(r0 + i) + (long long)(r0 + l) * J.R];
  }
  __syncthreads();
  for (int j = 0; j < w; ++j) {
    T* x = P + (long long)j * nr;
    if (warp == 0) {
      double s2 = 0.0;
      for (int i = j + 1 + lane; i < nr; i += 32) s2 += cabs2(x[i]);
      s2 = wsum(s2);
      const T alpha = x[j];
      T tau = czero<T>();
      const bool refl = s2 > 0.0 || cim(alpha) != 0.0;
      double beta = 0.0;
      if (refl) {
        beta = -copysign(sqrt(cabs2(alpha) + s2), cre(alpha));
        tau = cmake<T>((beta - cre(alpha)) / beta, -cim(alpha) / beta);
        // 1 / (alpha - beta)
        T scale;
        if constexpr (CPLX) {
          const double dr = alpha.x - beta, di = alpha.y, dd = 1.0 / (dr * dr + di * di);
          scale = make_double2(dr * dd, -di * dd);
        } else {
          scale = 1.0 / (alpha - beta);
        }
        for (int i = j + 1 + lane; i < nr; i += 32) x[i] = cmul(x[i], scale);
      }
      __syncwarp();
      if (lane == 0) {
        tau_sh[j] = tau;
        if (refl) x[j] = cmake<T>(beta, 0.0);
      }
    }
    __syncthreads();
    const T tau = tau_sh[j];
    if (warp < w - 1 - j && cabs2(tau) != 0.0) {
      T* y = P + (long long)(j + 1 + warp) * nr;
      T d = lane == 0 ? y[j] : czero<T>();   // v_j = 1
      for (int i = j + 1 + lane; i < nr; i += 32) d = cadd(d, cj_mul(x[i], y[i]));
      d = wsum_t(d);
      const T f = cmul(cconj(tau), d);
      if (lane == 0) y[j] = csub(y[j], f);
      for (int i = j + 1 + lane; i < nr; i += 32) y[i] = csub(y[i], cmul(x[i], f));
    }
    __syncthreads();
  }
  // S(q, j) = v_q^H v_j for q < j (rows j .. nr-1; v_j(j) = 1, v_q(j) = P(j, q))
  for (int pr = warp; pr < w * w; pr += kSvdWarps) {
    const int q = pr / w, j = pr % w;
    if (q >= j) continue;
    const T* vq = P + (long long)q * nr;
    const T* vj = P + (long long)j * nr;
    T d = lane == 0 ? cconj(vq[j]) : czero<T>();
    for (int i = j + 1 + lane; i < nr; i += 32) d = cadd(d, cj_mul(vq[i], vj[i]));
    d = wsum_t(d);
    if (lane == 0) S_sh[q + j * NB] = d;
  }
  __syncthreads();
  // T: T(j, j) = tau_j, T(0:j, j) = -tau_j T(0:j, 0:j) S(0:j, j)
  T* Tm = static_cast<T*>(qbuf) + J.toff + (long long)k * NB * NB;
  if (warp == 0) {
    __shared__ T T_sh[NB * NB];
    for (int e = lane; e < NB * NB; e += 32) T_sh[e] = czero<T>();
    __syncwarp();
    for (int j = 0; j < w; ++j) {
      const T tj = tau_sh[j];
      T v = czero<T>();
      if (lane < j) {
        for (int q = lane; q < j; ++q) v = cadd(v, cmul(T_sh[lane + q * NB], S_sh[q + j * NB]));
        v = cmul(cscale(tj, -1.0), v);
      }
      __syncwarp();
      if (lane < j) T_sh[lane + j * NB] = v;
      if (lane == j) T_sh[j + j * NB] = tj;
      __syncwarp();
    }
    for (int e = lane; e < NB * NB; e += 32) Tm[e] = T_sh[e];
  }
  for (int e = tid; e < nr * w; e += blockDim.x) {
    const int i = e % nr, l = e / nr;
    A[(r0 + i) + (long long)(r0 + l) * J.R] = P[e];
  }
  __syncthreads();   // P, tau_sh and S_sh are reused by the next panel this CTA takes
}

// X(r0:R, c1:c1+tw) <- H X with H = I - Y T Y^H (adj = 0) or H^H = I - Y T^H Y^H
// (adj = 1), Y = the unit lower trapezoidal reflectors of panel k.  Two passes
// over row chunks: Z = T' (Y^H X), then X -= Y Z (a single chunk stays in shared
// memory between the passes).
template <bool CPLX>
__device__ void qr_apply_tile(const QrJob& J, int k, int c1, int ncols, int adj, const void* qbuf, void* xbase,
                              long long xoff, unsigned char* smem) {
  using T = typename SvdT<CPLX>::T;
  using Gm = QrGeom<CPLX>;
  constexpr int NB = Gm::NB, RC = Gm::RC, LD = Gm::LD, NT = Gm::NT, G = Gm::G;
  const int r0 = k * NB, nr = J.R - r0, w = min(NB, J.C - r0), tw = min(NB, ncols - c1);
  const T* A = static_cast<const T*>(qbuf) + J.qoff;
  const T* Tm = static_cast<const T*>(qbuf) + J.toff + (long long)k * NB * NB;
  T* X = static_cast<T*>(xbase) + xoff;
  T* Vs = reinterpret_cast<T*>(smem);      // RC x NB (ld LD)
  T* Xs = Vs + LD * NB;                    // RC x NB (ld LD)
  T* Yp = Xs + LD * NB;                    // G partial sums of Y (NB x NB each)
  T* Zs = Yp + G * NT;                     // Z (NB x NB)
  const int tid = threadIdx.x;
  const int g = tid / NT, l = (tid % NT) / NB, t = tid % NB;
  const int nch = (nr + RC - 1) / RC;
  auto load = [&](int rr0, int rows) {
    for (int e = tid; e < RC * NB; e += kSvdThreads) {
      const int i = e % RC, c = e / RC, gi = rr0 + i;
      T v = czero<T>(), x = czero<T>();
      if (i < rows) {
        if (c < w) v = gi < c ? czero<T>() : (gi == c ? cmake<T>(1.0, 0.0) : A[(r0 + gi) + (long long)(r0 + c) * J.R]);
        if (c < tw) x = X[(r0 + gi) + (long long)(c1 + c) * J.R];
      }
      Vs[i + c * LD] = v;
      Xs[i + c * LD] = x;
    }
  };
  T acc = czero<T>();
  for (int ch = 0; ch < nch; ++ch) {
    const int rr0 = ch * RC, rows = min(RC, nr - rr0);
    load(rr0, rows);
    __syncthreads();
    for (int i = g; i < rows; i += G) acc = cadd(acc, cj_mul(Vs[i + l * LD], Xs[i + t * LD]));
    __syncthreads();
  }
  Yp[g * NT + l * NB + t] = acc;
  __syncthreads();
  if (tid < NT) {
    T y = czero<T>();
    for (int q = 0; q < G; ++q) y = cadd(y, Yp[q * NT + l * NB + t]);
    Zs[l * NB + t] = y;   // Y(l, t), row-major
  }
  __syncthreads();
  T z = czero<T>();
  if (tid < NT) {
    // Z(l, t) = sum_q T'(l, q) Y(q, t), T' = T (upper) or T^H (lower)
    for (int q = 0; q < w; ++q) {
      const T tq = adj ? cconj(Tm[q + l * NB]) : Tm[l + q * NB];
      z = cadd(z, cmul(tq, Zs[q * NB + t]));
    }
  }
  __syncthreads();
  if (tid < NT) Zs[l * NB + t] = z;
  __syncthreads();
  for (int ch = 0; ch < nch; ++ch) {
    const int rr0 = ch * RC, rows = min(RC, nr - rr0);
    if (nch > 1) {
      load(rr0, rows);
      __syncthreads();
    }
    for (int e = tid; e < RC * NB; e += kSvdThreads) {
      const int i = e % RC, c = e / RC;
      if (i >= rows || c >= tw) continue;
      T x = Xs[i + c * LD];
#pragma unroll
      for (int q = 0; q < NB; ++q) x = csub(x, cmul(Vs[i + q * LD], Zs[q * NB + c]));
      X[(r0 + rr0 + i) + (long long)(c1 + c) * J.R] = x;
    }
    __syncthreads();
  }
}

template <bool CPLX>
constexpr size_t qr_tile_smem() {
  using Gm = QrGeom<CPLX>;
  return (size_t)(2 * Gm::LD * Gm::NB + Gm::G * Gm::NT + Gm::NT) * (CPLX ? 16 : 8);
}

// The blocked QR of every job: step k factors panel k of every job that has one,
// then updates every NB-column tile right of it; a bounded grid barrier after
// each phase.
template <bool CPLX>
__global__ void __launch_bounds__(kSvdThreads) qr_coop_kernel(const QrJob* __restrict__ jobs,
                                                              const int* __restrict__ panels, const int* __restrict__ poff,
                                                              const QrTile* __restrict__ tiles, const int* __restrict__ toff,
                                                              int steps, void* qbuf, SvdCtl* ctl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->t0 = svd_gtime();
  for (int k = 0; k < steps; ++k) {
    for (int p = poff[k] + blockIdx.x; p < poff[k + 1]; p += gridDim.x) qr_panel<CPLX>(jobs[panels[p]], k, qbuf, smem_raw);
    if (!svd_grid_sync(ctl)) return;
    for (int t = toff[k] + blockIdx.x; t < toff[k + 1]; t += gridDim.x) {
      const QrTile tl = tiles[t];
      const QrJob& J = jobs[tl.job];
      qr_apply_tile<CPLX>(J, k, tl.c1, J.C, 1, qbuf, qbuf, J.qoff, smem_raw);
    }
    if (!svd_grid_sync(ctl)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->t1 = svd_gtime();
}

// X <- Q X for every job: its block reflectors applied from the last panel to
// the first to X (R x C at woff, in the output W or in the QR buffer).
template <bool CPLX>
__global__ void __launch_bounds__(kSvdThreads) qr_unmq_kernel(const QrJob* __restrict__ jobs,
                                                              const QrTile* __restrict__ tiles, const int* __restrict__ toff,
                                                              int steps, void* qbuf, void* out, SvdCtl* ctl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->t0 = svd_gtime();
  for (int k = steps - 1; k >= 0; --k) {
    for (int t = toff[k] + blockIdx.x; t < toff[k + 1]; t += gridDim.x) {
      const QrTile tl = tiles[t];
      const QrJob& J = jobs[tl.job];
      qr_apply_tile<CPLX>(J, k, tl.c1, J.C, 0, qbuf, J.x_in_q ? qbuf : out, J.woff, smem_raw);
    }
    if (k > 0 && !svd_grid_sync(ctl)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->t1 = svd_gtime();
}

// R^H (lower triangular, C x C) of src's factor into dst's matrix to factor
// (to_jacobi = 0), or into dst's Jacobi W with V = I (to_jacobi = 1).
template <bool CPLX>
__global__ void qr_rh_kernel(const QrJob* src, const QrJob* dst, void* qbuf, int to_jacobi) {
  using T = typename SvdT<CPLX>::T;
  const QrJob S = src[blockIdx.x], D = dst[blockIdx.x];
  const T* A = static_cast<const T*>(qbuf) + S.qoff;
  T* W = static_cast<T*>(qbuf) + (to_jacobi ? D.jwoff : D.qoff);
  T* V = static_cast<T*>(qbuf) + D.jvoff;
  const int C = S.C;
  for (long long e = threadIdx.x + (long long)blockIdx.y * blockDim.x; e < (long long)C * C;
       e += (long long)blockDim.x * gridDim.y) {
    const int r = (int)(e % C), c = (int)(e / C);
    W[e] = r >= c ? cconj(A[c + (long long)r * S.R]) : czero<T>();
    if (to_jacobi) V[e] = cmake<T>(r == c ? 1.0 : 0.0, 0.0);
  }
}

// Before the Q applications: the output W = [R1^H V2; 0] (R x C).
template <bool CPLX>
__global__ void qr_wout_kernel(const QrJob* jobs, const void* qbuf, void* work) {
  using T = typename SvdT<CPLX>::T;
  const QrJob J = jobs[blockIdx.x];
  const T* Wj = static_cast<const T*>(qbuf) + J.jwoff;
  T* W = static_cast<T*>(work) + J.woff;
  for (long long e = threadIdx.x + (long long)blockIdx.y * blockDim.x; e < (long long)J.R * J.C;
       e += (long long)blockDim.x * gridDim.y) {
    const int r = (int)(e % J.R), c = (int)(e / J.R);
    W[e] = r < J.C ? Wj[r + (long long)c * J.C] : czero<T>();
  }
}

// After them: the output V = P (Q1 V2), rows put back in the order of op(A)'s columns.
template <bool CPLX>
__global__ void qr_vout_kernel(const QrJob* jobs, const void* qbuf, void* vmat, const int* perm) {
  using T = typename SvdT<CPLX>::T;
  const QrJob J = jobs[blockIdx.x];
  const T* Vj = static_cast<const T*>(qbuf) + J.jvoff;
  T* V = static_cast<T*>(vmat) + J.voff;
  const int* p = perm + J.soff;
  for (long long e = threadIdx.x + (long long)blockIdx.y * blockDim.x; e < (long long)J.C * J.C;
       e += (long long)blockDim.x * gridDim.y) {
    const int i = (int)(e % J.C), c = (int)(e / J.C);
    V[p[i] + (long long)c * J.C] = Vj[e];
  }
}

// Host driver.  Runs all sweeps in one cooperative launch when the device allows
// it, otherwise one launch per round and one host synchronisation per sweep to
// test convergence.  Returns the number of sweeps taken (or -1 when max_sweeps
// was reached).
template <bool CPLX, int B>
static int jacobi_run(const void* a, void* work, void* vmat, double* sv, const std::vector<SvdJob>& hjobs,
                      int max_sweeps, cudaStream_t s, double* kernel_ms, int copy = 1, int stream = 0) {
  const int nj = (int)hjobs.size();
  std::vector<int> bsz(nj), nblk(nj), nrounds(nj);
  int max_rounds = 0, maxR = 0;
  long long maxRC = 0;
  size_t smem = 0;
  for (int j = 0; j < nj; ++j) {
    const int R = hjobs[j].trans ? hjobs[j].n : hjobs[j].m;
    const int C = hjobs[j].trans ? hjobs[j].m : hjobs[j].n;
    maxR = std::max(maxR, R);
    maxRC = std::max<long long>(maxRC, (long long)R + C);
    bsz[j] = B;
    nblk[j] = (C + bsz[j] - 1) / bsz[j];
    const int N = nblk[j] + (nblk[j] & 1);
    nrounds[j] = nblk[j] <= 1 ? 1 : N - 1;
    max_rounds = std::max(max_rounds, nrounds[j]);
    smem = svd_smem_bytes<CPLX, B>();
  }
  // visits hold the pair's columns of W and V in shared memory when the largest fits
  const int res = !stream && svd_res_smem_bytes<CPLX, B>(maxRC) <= kSvdResMax ? 1 : 0;
  if (res) smem = std::max(smem, svd_res_smem_bytes<CPLX, B>(maxRC));
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
  jacobi_init_kernel<CPLX><<<ig, 256, 0, s>>>(djobs.as<SvdJob>(), a, work, vmat, dperm.as<int>(), copy);
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
    int resv = res;
    void* a_work = work;
    void* a_vmat = vmat;
    double* a_nrm = sv;   // column norms of each sweep; the final singular values overwrite them
    int* a_perm = dperm.as<int>();
    void* args[] = {(void*)&pj,     (void*)&njv,    (void*)&pp,   (void*)&pr, (void*)&mr,   (void*)&a_work,
                    (void*)&a_vmat, (void*)&a_nrm, (void*)&a_perm, (void*)&tolv, (void*)&pc, (void*)&pctl,
                    (void*)&ms, (void*)&resv};
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
                                                                work, vmat, dperm.as<int>(), tol, dcnt.as<int>(), res);
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

// Column blocks of the Jacobi for these jobs: 8 when the widest round of
// 16-column pairs would keep fewer than half the SMs busy, else 16.
static bool narrow_blocks(const std::vector<SvdJob>& hjobs) {
  int dev = 0, nsm = 0;
  SADMRG_CUDA(cudaGetDevice(&dev));
  SADMRG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  long long pairs16 = 0;
  for (const SvdJob& J : hjobs) {
    const int C = J.trans ? J.m : J.n;
    const int nb = (C + 15) / 16;
    pairs16 += nb <= 1 ? 1 : nb / 2;
  }
  return 2 * pairs16 < nsm;
}

// Launches a cooperative kernel on the largest grid the device keeps resident,
// capped at `want` CTAs.  Returns false (nothing launched) when it cannot.
static bool coop_launch(const void* fn, int want, size_t smem, void** args, cudaStream_t s) {
  int dev = 0, coop = 0, nsm = 0, per_sm = 0;
  SADMRG_CUDA(cudaGetDevice(&dev));
  SADMRG_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  SADMRG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  SADMRG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  SADMRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSvdThreads, smem));
  if (!coop || per_sm <= 0) return false;
  const int grid = std::max(1, std::min(want, per_sm * nsm));
  SADMRG_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kSvdThreads), args, smem, s));
  return true;
}

// Per-step work lists of a set of QrJobs: the panels and trailing tiles of the
// QR (qr_coop_kernel), or the tiles of a Q application (qr_unmq_kernel).
struct QrLists {
  std::vector<int> panels, poff, toff;
  std::vector<QrTile> tiles;
  int steps = 0, want = 1;
};
template <int NB>
static QrLists qr_lists(const std::vector<QrJob>& jobs, bool unmq) {
  QrLists L;
  for (const QrJob& J : jobs) L.steps = std::max(L.steps, (J.C + NB - 1) / NB);
  L.poff.assign(L.steps + 1, 0);
  L.toff.assign(L.steps + 1, 0);
  for (int k = 0; k < L.steps; ++k) {
    L.poff[k] = (int)L.panels.size();
    L.toff[k] = (int)L.tiles.size();
    for (int j = 0; j < (int)jobs.size(); ++j) {
      if (jobs[j].C <= k * NB) continue;
      if (!unmq) L.panels.push_back(j);
      for (int c1 = unmq ? 0 : (k + 1) * NB; c1 < jobs[j].C; c1 += NB) L.tiles.push_back({j, c1});
    }
    L.want = std::max({L.want, (int)L.panels.size() - L.poff[k], (int)L.tiles.size() - L.toff[k]});
  }
  L.poff[L.steps] = (int)L.panels.size();
  L.toff[L.steps] = (int)L.tiles.size();
  return L;
}

// Device copies of a job array and its lists, and the cooperative launch of the
// QR (unmq = false) or of the Q application (unmq = true).  Returns false when
// the device cannot run it cooperatively.
template <bool CPLX>
struct QrLaunch {
  DevBuf dj, dpan, dpoff, dtl, dtoff;
  QrLists L;
  bool run(const std::vector<QrJob>& jobs, bool unmq, void* qbuf, void* out, SvdCtl* ctl, cudaStream_t s) {
    constexpr int NB = QrGeom<CPLX>::NB;
    L = qr_lists<NB>(jobs, unmq);
    int maxR = 0;
    for (const QrJob& J : jobs) maxR = std::max(maxR, J.R);
    dj.alloc(sizeof(QrJob) * jobs.size(), s);
    dpan.alloc(sizeof(int) * std::max<size_t>(L.panels.size(), 1), s);
    dpoff.alloc(sizeof(int) * (L.steps + 1), s);
    dtl.alloc(sizeof(QrTile) * std::max<size_t>(L.tiles.size(), 1), s);
    dtoff.alloc(sizeof(int) * (L.steps + 1), s);
    SADMRG_CUDA(cudaMemcpyAsync(dj.get(), jobs.data(), sizeof(QrJob) * jobs.size(), cudaMemcpyHostToDevice, s));
    if (!L.panels.empty())
      SADMRG_CUDA(cudaMemcpyAsync(dpan.get(), L.panels.data(), sizeof(int) * L.panels.size(), cudaMemcpyHostToDevice, s));
    if (!L.tiles.empty())
      SADMRG_CUDA(cudaMemcpyAsync(dtl.get(), L.tiles.data(), sizeof(QrTile) * L.tiles.size(), cudaMemcpyHostToDevice, s));
    SADMRG_CUDA(cudaMemcpyAsync(dpoff.get(), L.poff.data(), sizeof(int) * (L.steps + 1), cudaMemcpyHostToDevice, s));
    SADMRG_CUDA(cudaMemcpyAsync(dtoff.get(), L.toff.data(), sizeof(int) * (L.steps + 1), cudaMemcpyHostToDevice, s));
    const QrJob* pj = dj.as<QrJob>();
    const int* pp = dpan.as<int>();
    const int* ppo = dpoff.as<int>();
    const QrTile* pt = dtl.as<QrTile>();
    const int* pto = dtoff.as<int>();
    int st = L.steps;
    void* qb = qbuf;
    void* o = out;
    SvdCtl* pc = ctl;
    if (unmq) {
      void* args[] = {(void*)&pj, (void*)&pt, (void*)&pto, (void*)&st, (void*)&qb, (void*)&o, (void*)&pc};
      return coop_launch((const void*)qr_unmq_kernel<CPLX>, L.want, qr_tile_smem<CPLX>(), args, s);
    }
    const size_t smem = std::max((size_t)maxR * NB * sizeof(typename SvdT<CPLX>::T), qr_tile_smem<CPLX>());
    void* args[] = {(void*)&pj, (void*)&pp, (void*)&ppo, (void*)&pt, (void*)&pto, (void*)&st, (void*)&qb, (void*)&pc};
    return coop_launch((const void*)qr_coop_kernel<CPLX>, L.want, smem, args, s);
  }
};

// The QR-preconditioned SVD (see the QR preconditioning notes above).  Returns
// the Jacobi sweeps (as jacobi_run), or 0 with *fallback set when the device
// cannot run the cooperative kernels (the call then runs without
// preconditioning).
template <bool CPLX>
static int qr_jacobi_run(const void* a, void* work, void* vmat, double* sv, const std::vector<SvdJob>& hjobs,
                         int max_sweeps, cudaStream_t s, double* kernel_ms, bool* fallback, int stream, int block) {
  using T = typename SvdT<CPLX>::T;
  constexpr int NB = QrGeom<CPLX>::NB;
  *fallback = false;
  const int nj = (int)hjobs.size();
  // q1: op(A) P = Q R (R x C); q2: R^H = Q1 R1 (C x C), whose Jacobi W = R1^H and V
  // live at jwoff / jvoff; the second Q application multiplies that V
  std::vector<QrJob> q1(nj), q2(nj);
  long long tot = 0, nsv = 1;
  for (int j = 0; j < nj; ++j) {
    const SvdJob& J = hjobs[j];
    const int R = std::max(J.m, J.n), C = std::min(J.m, J.n), np = (C + NB - 1) / NB;
    QrJob& A = q1[j];
    QrJob& B = q2[j];
    A = QrJob{};
    A.aoff = J.aoff; A.woff = J.woff; A.voff = J.voff; A.soff = J.soff;
    A.m = J.m; A.n = J.n; A.trans = J.trans; A.R = R; A.C = C; A.x_in_q = 0;
    A.qoff = tot;  tot += (long long)R * C;
    A.toff = tot;  tot += (long long)np * NB * NB;
    B = A;
    B.m = B.n = B.R = C; B.trans = 0;
    B.qoff = tot;  tot += (long long)C * C;
    B.toff = tot;  tot += (long long)np * NB * NB;
    A.jwoff = B.jwoff = tot; tot += (long long)C * C;
    A.jvoff = B.jvoff = tot; tot += (long long)C * C;
    B.woff = B.jvoff;   // the second Q application multiplies the Jacobi's V
    B.x_in_q = 1;
    nsv = std::max<long long>(nsv, J.soff + C);
  }
  DevBuf qbuf(sizeof(T) * std::max<long long>(tot, 1), s), dperm(sizeof(int) * nsv, s), dctl(3 * sizeof(SvdCtl), s);
  SADMRG_CUDA(cudaMemsetAsync(dctl.get(), 0, 3 * sizeof(SvdCtl), s));
  SvdCtl* ctl = dctl.as<SvdCtl>();
  QrLaunch<CPLX> L1, L2, LU;
  // P and W0 = op(A) P need the job array on the device: the first QR's copy
  L1.dj.alloc(sizeof(QrJob) * nj, s);
  SADMRG_CUDA(cudaMemcpyAsync(L1.dj.get(), q1.data(), sizeof(QrJob) * nj, cudaMemcpyHostToDevice, s));
  qr_order_kernel<CPLX><<<nj, kSvdThreads, 0, s>>>(static_cast<const QrJob*>(L1.dj.get()), a, sv, dperm.as<int>());
  qr_gather_kernel<CPLX><<<dim3(nj, 32), 256, 0, s>>>(static_cast<const QrJob*>(L1.dj.get()), a, qbuf.get(), dperm.as<int>());
  SADMRG_CUDA(cudaGetLastError());
  if (!L1.run(q1, false, qbuf.get(), work, ctl, s)) {
    *fallback = true;
    return 0;
  }
  L2.dj.alloc(sizeof(QrJob) * nj, s);
  SADMRG_CUDA(cudaMemcpyAsync(L2.dj.get(), q2.data(), sizeof(QrJob) * nj, cudaMemcpyHostToDevice, s));
  qr_rh_kernel<CPLX><<<dim3(nj, 16), 256, 0, s>>>(static_cast<const QrJob*>(L1.dj.get()), static_cast<const QrJob*>(L2.dj.get()), qbuf.get(), 0);
  SADMRG_CUDA(cudaGetLastError());
  SADMRG_REQUIRE(L2.run(q2, false, qbuf.get(), work, ctl + 1, s), SADMRG_ERR_CUDA,
                 "svd: the second cooperative QR cannot be launched");
  qr_rh_kernel<CPLX><<<dim3(nj, 16), 256, 0, s>>>(static_cast<const QrJob*>(L2.dj.get()), static_cast<const QrJob*>(L2.dj.get()), qbuf.get(), 1);
  SADMRG_CUDA(cudaGetLastError());
  // the Jacobi on R1^H (C x C, W and V in qbuf)
  std::vector<SvdJob> jj(nj);
  for (int j = 0; j < nj; ++j) {
    SvdJob& J = jj[j];
    J.aoff = 0;
    J.woff = q2[j].jwoff;
    J.voff = q2[j].jvoff;
    J.soff = q2[j].soff;
    J.m = J.n = q2[j].C;
    J.trans = 0;
  }
  double jms = -1.0;
  const bool narrow = block == 8 || (block == 0 && narrow_blocks(jj));
  const int sweeps = narrow
                         ? jacobi_run<CPLX, 8>(nullptr, qbuf.get(), qbuf.get(), sv, jj, max_sweeps, s, &jms, 0, stream)
                         : jacobi_run<CPLX, 16>(nullptr, qbuf.get(), qbuf.get(), sv, jj, max_sweeps, s, &jms, 0, stream);
  if (sweeps <= 0) return sweeps;
  // W = Q [R1^H V2; 0] and Q1 V2, both Q applications in one launch, then V = P (Q1 V2)
  qr_wout_kernel<CPLX><<<dim3(nj, 16), 256, 0, s>>>(static_cast<const QrJob*>(L1.dj.get()), qbuf.get(), work);
  SADMRG_CUDA(cudaGetLastError());
  std::vector<QrJob> qu(q1);
  qu.insert(qu.end(), q2.begin(), q2.end());
  SADMRG_REQUIRE(LU.run(qu, true, qbuf.get(), work, ctl + 2, s), SADMRG_ERR_CUDA,
                 "svd: the cooperative Q application cannot be launched");
  qr_vout_kernel<CPLX><<<dim3(nj, 16), 256, 0, s>>>(static_cast<const QrJob*>(L1.dj.get()), qbuf.get(), vmat, dperm.as<int>());
  SADMRG_CUDA(cudaGetLastError());
  SvdCtl hctl[3];
  SADMRG_CUDA(cudaMemcpyAsync(hctl, dctl.get(), 3 * sizeof(SvdCtl), cudaMemcpyDeviceToHost, s));
  SADMRG_CUDA(cudaStreamSynchronize(s));
  SADMRG_REQUIRE(hctl[0].status == 0 && hctl[1].status == 0 && hctl[2].status == 0, SADMRG_ERR_CUDA,
                 "svd: a grid barrier of the QR preconditioning ran out of time");
  if (kernel_ms && jms >= 0.0) {
    *kernel_ms = jms;
    for (const SvdCtl& c : hctl) *kernel_ms += (double)(c.t1 - c.t0) * 1e-6;
  }
  return sweeps;
}

int run_jacobi_svd(bool cplx, const void* a, void* work, void* vmat, double* sv, const std::vector<SvdJob>& hjobs,
                   int max_sweeps, cudaStream_t s, double* kernel_ms, int precondition, int stream, int block) {
  if (kernel_ms) *kernel_ms = -1.0;
  if (hjobs.empty()) return 0;
  if (precondition) {
    // the panel of the tallest block must fit in shared memory
    int maxR = 0, maxC = 0;
    for (const SvdJob& J : hjobs) {
      maxR = std::max(maxR, std::max(J.m, J.n));
      maxC = std::max(maxC, std::min(J.m, J.n));
    }
    const size_t panel = (size_t)maxR * (cplx ? QrGeom<true>::NB * 16 : QrGeom<false>::NB * 8);
    if (panel <= kQrSmemMax && (maxC >= kQrMinCols || precondition == 2)) {
      bool fallback = false;
      const int sw = cplx ? qr_jacobi_run<true>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms, &fallback, stream, block)
                          : qr_jacobi_run<false>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms, &fallback, stream, block);
      if (!fallback) return sw;
    }
  }
  // column blocks of 16, or of 8 when the widest round of 16-column pairs would
  // keep fewer than half the SMs busy: narrower pairs double the CTAs per round
  // and cut each visit's work to a quarter, which wins while SMs are idle (D=512:
  // 1.87 -> 1.65 s of SVD per sweep) and loses once they are not (complex D=2048:
  // 4.8 -> 5.5 s per iDMRG)
  const bool narrow = block == 8 || (block == 0 && narrow_blocks(hjobs));
  if (cplx)
    return narrow ? jacobi_run<true, 8>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms, 1, stream)
                  : jacobi_run<true, 16>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms, 1, stream);
  return narrow ? jacobi_run<false, 8>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms, 1, stream)
                : jacobi_run<false, 16>(a, work, vmat, sv, hjobs, max_sweeps, s, kernel_ms, 1, stream);
}

}  // namespace sadmrg
