// gemm_tf32x3.cu -- split-precision (3xTF32) grouped GEMM.
//
// Each FP64 operand x is rounded to FP32 and split as x ~ hi + lo with
// hi = tf32(x), lo = tf32(x - hi); a product is hi*hi + hi*lo + lo*hi (the
// lo*lo term is below FP32 resolution), the "3xTF32" scheme of Markidis et al.
// (2018) and Ootomo & Yokota (2022).  Tensor-core partial sums are FP32 and are
// folded into FP64 register accumulators after every task term, so long
// accumulation lists lose no more than one FP32 rounding per term.  Complex
// operands run as real/imaginary splits (rr, ii, ri + ir).
#include <cuda_runtime.h>
#include <cstdint>

#include "kernels.cuh"

namespace sadmrg {

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

// D(16x8) += A(16x8, row) * B(8x8, col), tf32 inputs, f32 accumulators
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ void mma3(float (&d)[4], const uint32_t (&ah)[4], const uint32_t (&al)[4],
                                     const uint32_t (&bh)[2], const uint32_t (&bl)[2]) {
  mma_tf32(d, al, bh);
  mma_tf32(d, ah, bl);
  mma_tf32(d, ah, bh);
}

constexpr int kT3Threads = 128;

template <bool CPLX, int BM, int BN, int BK>
__global__ void __launch_bounds__(kT3Threads) grouped_gemm_tf32x3(const GemmTerm* __restrict__ terms,
                                                                   const GemmJob* __restrict__ jobs,
                                                                   const GemmTile* __restrict__ tiles, Bases bases) {
  constexpr int PAD = 8;
  constexpr int NP = CPLX ? 2 : 1;  // planes (re, im)
  __shared__ uint32_t Ah[NP][BK][BM + PAD], Al[NP][BK][BM + PAD];
  __shared__ uint32_t Bh[NP][BK][BN + PAD], Bl[NP][BK][BN + PAD];
  const GemmTile t = tiles[blockIdx.x];
  const GemmJob J = jobs[t.job];
  const int row0 = t.tm * BM, col0 = t.tn * BN;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp >> 1, wn = warp & 1;
  const int g = lane >> 2, tg = lane & 3;
  constexpr int WM = BM / 2, WN = BN / 2, MT = WM / 16, NT = WN / 8;
  constexpr int NACC = CPLX ? 3 : 1;  // rr, ii, im
  double accd[NACC][MT][NT][4];
#pragma unroll
  for (int q = 0; q < NACC; ++q)
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) accd[q][i][j][e] = 0.0;

  for (int ti = 0; ti < J.nt; ++ti) {
    const GemmTerm T = terms[J.t0 + ti];
    const bool ta = T.flags & TF_TA, tb = T.flags & TF_TB;
    const double ca = (T.flags & TF_CA) ? -1.0 : 1.0, cb = (T.flags & TF_CB) ? -1.0 : 1.0;
    float acc[NACC][MT][NT][4];
#pragma unroll
    for (int q = 0; q < NACC; ++q)
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) acc[q][i][j][e] = 0.f;
    for (int k0 = 0; k0 < T.k; k0 += BK) {
      for (int e = tid; e < BM * BK; e += kT3Threads) {
        int i, kk;
        if (!ta) { i = e % BM; kk = e / BM; } else { kk = e % BK; i = e / BK; }
        const int gi = row0 + i, gk = k0 + kk;
        const long long idx = ta ? gk + (long long)gi * T.lda : gi + (long long)gk * T.lda;
        const bool in = gi < J.m && gk < T.k;
        if (CPLX) {
          double2 v = in ? (static_cast<const double2*>(bases.p[T.abuf]) + T.aoff)[idx] : make_double2(0.0, 0.0);
          v.y *= ca;
          split3(v.x * T.ar - v.y * T.ai, Ah[0][kk][i], Al[0][kk][i]);
          split3(v.x * T.ai + v.y * T.ar, Ah[NP - 1][kk][i], Al[NP - 1][kk][i]);
        } else {
          const double v = in ? (static_cast<const double*>(bases.p[T.abuf]) + T.aoff)[idx] : 0.0;
          split3(v * T.ar, Ah[0][kk][i], Al[0][kk][i]);
        }
      }
      for (int e = tid; e < BK * BN; e += kT3Threads) {
        int j, kk;
        if (!tb) { kk = e % BK; j = e / BK; } else { j = e % BN; kk = e / BN; }
        const int gj = col0 + j, gk = k0 + kk;
        const long long idx = tb ? gj + (long long)gk * T.ldb : gk + (long long)gj * T.ldb;
        const bool in = gj < J.n && gk < T.k;
        if (CPLX) {
          const double2 v = in ? (static_cast<const double2*>(bases.p[T.bbuf]) + T.boff)[idx] : make_double2(0.0, 0.0);
          split3(v.x, Bh[0][kk][j], Bl[0][kk][j]);
          split3(v.y * cb, Bh[NP - 1][kk][j], Bl[NP - 1][kk][j]);
        } else {
          const double v = in ? (static_cast<const double*>(bases.p[T.bbuf]) + T.boff)[idx] : 0.0;
          split3(v, Bh[0][kk][j], Bl[0][kk][j]);
        }
      }
      __syncthreads();
#pragma unroll
      for (int k8 = 0; k8 < BK; k8 += 8) {
        uint32_t ah[NP][MT][4], al[NP][MT][4], bh[NP][NT][2], bl[NP][NT][2];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
#pragma unroll
          for (int mi = 0; mi < MT; ++mi) {
            const int r = wm * WM + mi * 16 + g;
            ah[p][mi][0] = Ah[p][k8 + tg][r];     al[p][mi][0] = Al[p][k8 + tg][r];
            ah[p][mi][1] = Ah[p][k8 + tg][r + 8]; al[p][mi][1] = Al[p][k8 + tg][r + 8];
            ah[p][mi][2] = Ah[p][k8 + tg + 4][r]; al[p][mi][2] = Al[p][k8 + tg + 4][r];
            ah[p][mi][3] = Ah[p][k8 + tg + 4][r + 8]; al[p][mi][3] = Al[p][k8 + tg + 4][r + 8];
          }
#pragma unroll
          for (int ni = 0; ni < NT; ++ni) {
            const int c = wn * WN + ni * 8 + g;
            bh[p][ni][0] = Bh[p][k8 + tg][c];     bl[p][ni][0] = Bl[p][k8 + tg][c];
            bh[p][ni][1] = Bh[p][k8 + tg + 4][c]; bl[p][ni][1] = Bl[p][k8 + tg + 4][c];
          }
        }
#pragma unroll
        for (int mi = 0; mi < MT; ++mi)
#pragma unroll
          for (int ni = 0; ni < NT; ++ni) {
            if (CPLX) {
              mma3(acc[0][mi][ni], ah[0][mi], al[0][mi], bh[0][ni], bl[0][ni]);          // re*re
              mma3(acc[1][mi][ni], ah[1][mi], al[1][mi], bh[1][ni], bl[1][ni]);          // im*im
              mma3(acc[NACC - 1][mi][ni], ah[0][mi], al[0][mi], bh[1][ni], bl[1][ni]);   // re*im
              mma3(acc[NACC - 1][mi][ni], ah[1][mi], al[1][mi], bh[0][ni], bl[0][ni]);   // im*re
            } else {
              mma3(acc[0][mi][ni], ah[0][mi], al[0][mi], bh[0][ni], bl[0][ni]);
            }
          }
      }
      __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < NACC; ++q)
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) accd[q][i][j][e] += (double)acc[q][i][j][e];
  }
  const bool accum = J.flags & JF_ACCUM;
#pragma unroll
  for (int mi = 0; mi < MT; ++mi)
#pragma unroll
    for (int ni = 0; ni < NT; ++ni)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = row0 + wm * WM + mi * 16 + g + (e >= 2 ? 8 : 0);
        const int c = col0 + wn * WN + ni * 8 + 2 * tg + (e & 1);
        if (r < J.m && c < J.n) {
          const long long idx = r + (long long)c * J.ldc;
          if (CPLX) {
            double2* C = static_cast<double2*>(bases.p[J.cbuf]) + J.coff;
            double2 v = make_double2(accd[0][mi][ni][e] - accd[1][mi][ni][e], accd[NACC - 1][mi][ni][e]);
            if (accum) { const double2 o = C[idx]; v.x += o.x; v.y += o.y; }
            C[idx] = v;
          } else {
            double* C = static_cast<double*>(bases.p[J.cbuf]) + J.coff;
            C[idx] = accum ? C[idx] + accd[0][mi][ni][e] : accd[0][mi][ni][e];
          }
        }
      }
}

void launch_grouped_gemm_tf32x3(bool cplx, const GemmTerm* terms, const GemmJob* jobs, const GemmTile* tiles,
                                int ntiles, const Bases& b, cudaStream_t s) {
  if (cplx)
    grouped_gemm_tf32x3<true, 32, 32, 16><<<ntiles, kT3Threads, 0, s>>>(terms, jobs, tiles, b);
  else
    grouped_gemm_tf32x3<false, 64, 64, 16><<<ntiles, kT3Threads, 0, s>>>(terms, jobs, tiles, b);
}

}  // namespace sadmrg
