// kernels.cu -- sm_100a kernels for the two-site DMRG hot path.
//
//  (the grouped block-GEMM executor is in gemm.cu)
//  * block utilities (segment axpy, block transpose, fuse fill, SVD gather);
//  * Krylov vector kernels with deterministic two-pass reductions;
//  * one-sided (Hestenes) block Jacobi SVD, column blocks staged in shared
//    memory, rotations accumulated into a small matrix applied to V at the end.
#include <cuda_runtime.h>
#include <cstdio>

#include "kernels.cuh"

namespace sadmrg {

// --------------------------------------------------------------------------
// block utilities
template <bool CPLX>
__global__ void seg_axpy_kernel(void* y, const void* x, const Seg* segs) {
  const Seg sg = segs[blockIdx.x];
  const long long stride = (long long)blockDim.x * gridDim.y;
  for (long long i = (long long)blockIdx.y * blockDim.x + threadIdx.x; i < sg.n; i += stride) {
    if (CPLX) {
      const double2 v = static_cast<const double2*>(x)[sg.soff + i];
      double2& o = static_cast<double2*>(y)[sg.doff + i];
      o.x += v.x * sg.ar - v.y * sg.ai;
      o.y += v.x * sg.ai + v.y * sg.ar;
    } else {
      static_cast<double*>(y)[sg.doff + i] += sg.ar * static_cast<const double*>(x)[sg.soff + i];
    }
  }
}

void launch_seg_axpy(bool cplx, void* y, const void* x, const Seg* segs, int nseg, cudaStream_t s) {
  if (nseg <= 0) return;
  dim3 grid(nseg, 16);
  if (cplx) seg_axpy_kernel<true><<<grid, 256, 0, s>>>(y, x, segs);
  else seg_axpy_kernel<false><<<grid, 256, 0, s>>>(y, x, segs);
}

template <class T>
__global__ void block_transpose_kernel(T* dst, const T* src, const Transp* jobs) {
  __shared__ T tile[32][33];
  const Transp tj = jobs[blockIdx.x];
  const int tr = (tj.rows + 31) / 32, tc = (tj.cols + 31) / 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int tIdx = blockIdx.y; tIdx < tr * tc; tIdx += gridDim.y) {
    const int bi = (tIdx % tr) * 32, bj = (tIdx / tr) * 32;
    for (int k = ty; k < 32; k += 8) {
      const int r = bi + tx, c = bj + k;
      if (r < tj.rows && c < tj.cols) tile[k][tx] = src[tj.soff + r + (long long)c * tj.rows];
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
      const int r = bj + tx, c = bi + k;  // dst is cols x rows
      if (r < tj.cols && c < tj.rows) dst[tj.doff + r + (long long)c * tj.cols] = tile[tx][k];
    }
    __syncthreads();
  }
}

void launch_block_transpose(bool cplx, void* dst, const void* src, const Transp* t, int nt, cudaStream_t s) {
  if (nt <= 0) return;
  dim3 grid(nt, 32);
  if (cplx) block_transpose_kernel<double2><<<grid, 256, 0, s>>>((double2*)dst, (const double2*)src, t);
  else block_transpose_kernel<double><<<grid, 256, 0, s>>>((double*)dst, (const double*)src, t);
}

// leg permutation of 3-leg blocks: one block of threads per tensor block, every
// destination element gathered from its source position (the tensors this serves,
// projected lower states of an excited-state sweep, are small)
template <class T>
__global__ void permute3_kernel(T* dst, const T* src, const Perm3* jobs) {
  const Perm3 J = jobs[blockIdx.x];
  const long long nd0 = J.d[J.p[0]], nd1 = J.d[J.p[1]], n = (long long)J.d[0] * J.d[1] * J.d[2];
  const long long st[3] = {1, J.d[0], (long long)J.d[0] * J.d[1]};   // source strides
  for (long long e = threadIdx.x + (long long)blockIdx.y * blockDim.x; e < n; e += (long long)blockDim.x * gridDim.y) {
    const long long i0 = e % nd0, i1 = (e / nd0) % nd1, i2 = e / (nd0 * nd1);
    dst[J.doff + e] = src[J.soff + i0 * st[J.p[0]] + i1 * st[J.p[1]] + i2 * st[J.p[2]]];
  }
}

void launch_permute3(bool cplx, void* dst, const void* src, const Perm3* t, int nt, cudaStream_t s) {
  if (nt <= 0) return;
  dim3 grid(nt, 8);
  if (cplx) permute3_kernel<double2><<<grid, 256, 0, s>>>((double2*)dst, (const double2*)src, t);
  else permute3_kernel<double><<<grid, 256, 0, s>>>((double*)dst, (const double*)src, t);
}

template <bool CPLX>
__global__ void fuse_fill_kernel(void* data, const FuseFill* f) {
  const FuseFill ff = f[blockIdx.x];
  const long long plane = (long long)ff.d0 * ff.d1;
  for (long long e = threadIdx.x; e < plane; e += blockDim.x) {
    const int a = (int)(e % ff.d0), b = (int)(e / ff.d0);
    const long long idx = ff.off + a + (long long)b * ff.d0 + (long long)(ff.pos + b * ff.d0 + a) * plane;
    if (CPLX) static_cast<double2*>(data)[idx] = make_double2(1.0, 0.0);
    else static_cast<double*>(data)[idx] = 1.0;
  }
}

void launch_fuse_fill(bool cplx, void* data, const FuseFill* f, int nf, cudaStream_t s) {
  if (nf <= 0) return;
  if (cplx) fuse_fill_kernel<true><<<nf, 256, 0, s>>>(data, f);
  else fuse_fill_kernel<false><<<nf, 256, 0, s>>>(data, f);
}

template <bool CPLX>
__global__ void gather_kernel(void* dst, const void* src, const double* w, const int* perm, const Gather* g) {
  const Gather G = g[blockIdx.x];
  const long long total = (long long)G.rows * G.kept;
  for (long long e = (long long)blockIdx.y * blockDim.x + threadIdx.x; e < total; e += (long long)blockDim.x * gridDim.y) {
    const int r = (int)(e % G.rows), c = (int)(e / G.rows);
    const double wv = w[G.woff + c];
    double sc = 1.0;
    if (G.p != 0.0) sc = (wv > 0.0) ? pow(wv, G.p) : 0.0;
    const long long si = G.soff + r + (long long)perm[G.poff + c] * G.lds;
    if (CPLX) {
      double2 v = static_cast<const double2*>(src)[si];
      if (G.conj) v.y = -v.y;
      v.x *= sc; v.y *= sc;
      static_cast<double2*>(dst)[G.doff + e] = v;
    } else {
      static_cast<double*>(dst)[G.doff + e] = static_cast<const double*>(src)[si] * sc;
    }
  }
}

void launch_gather(bool cplx, void* dst, const void* src, const double* w, const int* perm, const Gather* g, int ng,
                   cudaStream_t s) {
  if (ng <= 0) return;
  dim3 grid(ng, 8);
  if (cplx) gather_kernel<true><<<grid, 256, 0, s>>>(dst, src, w, perm, g);
  else gather_kernel<false><<<grid, 256, 0, s>>>(dst, src, w, perm, g);
}

template <bool CPLX>
__global__ void scale_kernel(void* x, double ar, double ai, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)blockDim.x * gridDim.x) {
    if (CPLX) {
      const double2 v = static_cast<double2*>(x)[i];
      static_cast<double2*>(x)[i] = make_double2(v.x * ar - v.y * ai, v.x * ai + v.y * ar);
    } else {
      static_cast<double*>(x)[i] *= ar;
    }
  }
}

void launch_scale(bool cplx, void* x, double ar, double ai, long long n, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)min((n + 255) / 256, 148LL * 8);
  if (cplx) scale_kernel<true><<<blocks, 256, 0, s>>>(x, ar, ai, n);
  else scale_kernel<false><<<blocks, 256, 0, s>>>(x, ar, ai, n);
}

// Reads bytes (a multiple of 16) of x; writes sink only when the xor of all
// words is a value no data here holds in practice, so the loads cannot be dropped.
__global__ void read_kernel(const uint4* __restrict__ x, long long n16, unsigned* sink) {
  unsigned acc = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (long long)blockDim.x * gridDim.x) {
    const uint4 v = __ldcg(x + i);
    acc ^= v.x ^ v.y ^ v.z ^ v.w;
  }
  if (acc == 0x9e3779b9u && sink) *sink = acc;
}

void launch_read(const void* x, long long bytes, unsigned* sink, cudaStream_t s) {
  if (bytes < 16) return;
  read_kernel<<<148 * 8, 256, 0, s>>>(static_cast<const uint4*>(x), bytes / 16, sink);
}

template <bool CPLX>
__global__ void fill_kernel(void* x, double vr, double vi, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)blockDim.x * gridDim.x) {
    if (CPLX) static_cast<double2*>(x)[i] = make_double2(vr, vi);
    else static_cast<double*>(x)[i] = vr;
  }
}

void launch_fill(bool cplx, void* x, double vr, double vi, long long n, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)min((n + 255) / 256, 148LL * 8);
  if (cplx) fill_kernel<true><<<blocks, 256, 0, s>>>(x, vr, vi, n);
  else fill_kernel<false><<<blocks, 256, 0, s>>>(x, vr, vi, n);
}

template <bool CPLX>
__device__ __forceinline__ void lanczos_scalar_op(int op, const void* dot, const double* beta_prev, void* out) {
  const double re = CPLX ? static_cast<const double2*>(dot)[0].x : static_cast<const double*>(dot)[0];
  if (op == 0) {
    if (CPLX) {
      static_cast<double2*>(out)[0] = make_double2(beta_prev[0], 0.0);
      static_cast<double2*>(out)[1] = make_double2(re, 0.0);
    } else {
      static_cast<double*>(out)[0] = beta_prev[0];
      static_cast<double*>(out)[1] = re;
    }
  } else {
    static_cast<double*>(out)[0] = sqrt(fabs(re));
  }
}

// --------------------------------------------------------------------------
// Krylov vector kernels
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// <V_j|x> in one launch: every block writes its partial sums, and the last block
// to finish (atomic count) adds them up -- one warp per dot, lane l taking
// partials l, l + 32, ... and the warp summing in a fixed tree, so the result
// does not depend on which block is last -- and, if op >= 0, applies the Krylov
// scalar step of lanczos_scalar_kernel to out[0].  counter is zero between launches.
template <bool CPLX>
__global__ void multi_dot_fused(const void* V, long long ldv, int nv, const void* x, long long n, double* partial,
                                void* out, unsigned* counter, int op, const double* beta_prev, void* sout) {
  constexpr int kG = 8;                 // dots per pass over the block's range
  __shared__ double red[2][kG][32];
  __shared__ int last;
  const long long per = (n + gridDim.x - 1) / gridDim.x;
  const long long lo = per * blockIdx.x, hi = min(n, lo + per);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j0 = 0; j0 < nv; j0 += kG) {
    const int g = min(kG, nv - j0);
    double sr[kG], si[kG];
#pragma unroll
    for (int u = 0; u < kG; ++u) { sr[u] = 0.0; si[u] = 0.0; }
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      if (CPLX) {
        const double2 b = static_cast<const double2*>(x)[i];
#pragma unroll
        for (int u = 0; u < kG; ++u)
          if (u < g) {
            const double2 a = static_cast<const double2*>(V)[(j0 + u) * ldv + i];
            sr[u] += a.x * b.x + a.y * b.y;  // conj(a) * b
            si[u] += a.x * b.y - a.y * b.x;
          }
      } else {
        const double b = static_cast<const double*>(x)[i];
#pragma unroll
        for (int u = 0; u < kG; ++u)
          if (u < g) sr[u] += static_cast<const double*>(V)[(j0 + u) * ldv + i] * b;
      }
    }
#pragma unroll
    for (int u = 0; u < kG; ++u) {
      if (u >= g) break;
      const double a = warp_sum(sr[u]);
      const double b = CPLX ? warp_sum(si[u]) : 0.0;
      if (l == 0) { red[0][u][w] = a; red[1][u][w] = b; }
    }
    __syncthreads();
    if (w < g) {   // warp u adds up dot j0 + u over the block's warps
      double a = (l < nw) ? red[0][w][l] : 0.0, b = (l < nw) ? red[1][w][l] : 0.0;
      a = warp_sum(a);
      if (CPLX) b = warp_sum(b);
      if (l == 0) {
        partial[(blockIdx.x * (long long)nv + j0 + w) * 2 + 0] = a;
        partial[(blockIdx.x * (long long)nv + j0 + w) * 2 + 1] = b;
      }
    }
    __syncthreads();
  }
  __threadfence();   // every writer's partials before the count
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int j = w; j < nv; j += nw) {
    double a = 0.0, b = 0.0;
    for (int p = l; p < (int)gridDim.x; p += 32) {
      a += __ldcg(partial + (p * (long long)nv + j) * 2 + 0);
      if (CPLX) b += __ldcg(partial + (p * (long long)nv + j) * 2 + 1);
    }
    a = warp_sum(a);
    if (CPLX) b = warp_sum(b);
    if (l == 0) {
      if (CPLX) static_cast<double2*>(out)[j] = make_double2(a, b);
      else static_cast<double*>(out)[j] = a;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (op >= 0) lanczos_scalar_op<CPLX>(op, out, beta_prev, sout);
    *counter = 0u;
  }
}

void launch_multi_dot(bool cplx, const void* V, long long ldv, int nv, const void* x, long long n, double* partial,
                      int npart, void* out, unsigned* counter, cudaStream_t s, int scalar_op, const double* beta_prev,
                      void* scalar_out) {
  if (nv <= 0) return;
  if (cplx)
    multi_dot_fused<true><<<npart, 256, 0, s>>>(V, ldv, nv, x, n, partial, out, counter, scalar_op, beta_prev,
                                               scalar_out);
  else
    multi_dot_fused<false><<<npart, 256, 0, s>>>(V, ldv, nv, x, n, partial, out, counter, scalar_op, beta_prev,
                                                scalar_out);
}

template <bool CPLX>
__global__ void multi_axpy_kernel(void* x, const void* V, long long ldv, int nv, const void* c, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)blockDim.x * gridDim.x) {
    if (CPLX) {
      double2 acc = static_cast<double2*>(x)[i];
      for (int j = 0; j < nv; ++j) {
        const double2 cj = static_cast<const double2*>(c)[j];
        const double2 v = static_cast<const double2*>(V)[j * ldv + i];
        acc.x -= cj.x * v.x - cj.y * v.y;
        acc.y -= cj.x * v.y + cj.y * v.x;
      }
      static_cast<double2*>(x)[i] = acc;
    } else {
      double acc = static_cast<double*>(x)[i];
      for (int j = 0; j < nv; ++j) acc -= static_cast<const double*>(c)[j] * static_cast<const double*>(V)[j * ldv + i];
      static_cast<double*>(x)[i] = acc;
    }
  }
}

void launch_multi_axpy(bool cplx, void* x, const void* V, long long ldv, int nv, const void* c, long long n,
                       cudaStream_t s) {
  if (nv <= 0 || n <= 0) return;
  const int blocks = (int)min((n + 255) / 256, 148LL * 8);
  if (cplx) multi_axpy_kernel<true><<<blocks, 256, 0, s>>>(x, V, ldv, nv, c, n);
  else multi_axpy_kernel<false><<<blocks, 256, 0, s>>>(x, V, ldv, nv, c, n);
}

template <bool CPLX>
__global__ void scale_inv_kernel(void* x, const double* scal, long long n) {
  const double inv = 1.0 / scal[0];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)blockDim.x * gridDim.x) {
    if (CPLX) { double2 v = static_cast<double2*>(x)[i]; v.x *= inv; v.y *= inv; static_cast<double2*>(x)[i] = v; }
    else static_cast<double*>(x)[i] *= inv;
  }
}

void launch_scale_inv(bool cplx, void* x, const double* scal, long long n, cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)min((n + 255) / 256, 148LL * 8);
  if (cplx) scale_inv_kernel<true><<<blocks, 256, 0, s>>>(x, scal, n);
  else scale_inv_kernel<false><<<blocks, 256, 0, s>>>(x, scal, n);
}

template <bool CPLX>
__global__ void lincomb_kernel(void* y, const void* V, long long ldv, int nv, const double* c, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)blockDim.x * gridDim.x) {
    if (CPLX) {
      double2 acc = make_double2(0.0, 0.0);
      for (int j = 0; j < nv; ++j) {
        const double2 v = static_cast<const double2*>(V)[j * ldv + i];
        acc.x += c[j] * v.x;
        acc.y += c[j] * v.y;
      }
      static_cast<double2*>(y)[i] = acc;
    } else {
      double acc = 0.0;
      for (int j = 0; j < nv; ++j) acc += c[j] * static_cast<const double*>(V)[j * ldv + i];
      static_cast<double*>(y)[i] = acc;
    }
  }
}

void launch_lincomb(bool cplx, void* y, const void* V, long long ldv, int nv, const double* c_dev, long long n,
                    cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)min((n + 255) / 256, 148LL * 8);
  if (cplx) lincomb_kernel<true><<<blocks, 256, 0, s>>>(y, V, ldv, nv, c_dev, n);
  else lincomb_kernel<false><<<blocks, 256, 0, s>>>(y, V, ldv, nv, c_dev, n);
}

}  // namespace sadmrg

// ---------------------------------------------------------------------------
// Segmented Krylov kernels for independent instances stored back to back:
// segment s is [seg[s], seg[s + 1]).  One block per segment, so every
// reduction runs in one fixed order (deterministic).
namespace sadmrg {

template <bool CPLX>
__global__ void __launch_bounds__(256) seg_multi_dot_kernel(const void* V, long long ldv, int nv, const void* x,
                                                            const long long* seg, void* out) {
  __shared__ double red[2][8];
  const int s = blockIdx.x;
  const long long lo = seg[s], hi = seg[s + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = 0; j < nv; ++j) {
    double sr = 0.0, si = 0.0;
    for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      if (CPLX) {
        const double2 a = static_cast<const double2*>(V)[j * ldv + i];
        const double2 b = static_cast<const double2*>(x)[i];
        sr += a.x * b.x + a.y * b.y;
        si += a.x * b.y - a.y * b.x;
      } else {
        sr += static_cast<const double*>(V)[j * ldv + i] * static_cast<const double*>(x)[i];
      }
    }
    sr = warp_sum(sr);
    if (CPLX) si = warp_sum(si);
    if (lane == 0) { red[0][warp] = sr; red[1][warp] = si; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += red[0][w]; b += red[1][w]; }
      if (CPLX) static_cast<double2*>(out)[(long long)s * nv + j] = make_double2(a, b);
      else static_cast<double*>(out)[(long long)s * nv + j] = a;
    }
    __syncthreads();
  }
}

void launch_seg_multi_dot(bool cplx, const void* V, long long ldv, int nv, const void* x, const long long* seg,
                          int nseg, void* out, cudaStream_t s) {
  if (nv <= 0 || nseg <= 0) return;
  if (cplx) seg_multi_dot_kernel<true><<<nseg, 256, 0, s>>>(V, ldv, nv, x, seg, out);
  else seg_multi_dot_kernel<false><<<nseg, 256, 0, s>>>(V, ldv, nv, x, seg, out);
}

// x -= sum_j c[s * cstride + j] V_j on segment s
template <bool CPLX>
__global__ void __launch_bounds__(256) seg_multi_axpy_kernel(void* x, const void* V, long long ldv, int nv,
                                                             const void* c, int cstride, const long long* seg) {
  const int s = blockIdx.x;
  const long long lo = seg[s], hi = seg[s + 1];
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    if (CPLX) {
      double2 acc = static_cast<double2*>(x)[i];
      for (int j = 0; j < nv; ++j) {
        const double2 cj = static_cast<const double2*>(c)[(long long)s * cstride + j];
        const double2 v = static_cast<const double2*>(V)[j * ldv + i];
        acc.x -= cj.x * v.x - cj.y * v.y;
        acc.y -= cj.x * v.y + cj.y * v.x;
      }
      static_cast<double2*>(x)[i] = acc;
    } else {
      double acc = static_cast<double*>(x)[i];
      for (int j = 0; j < nv; ++j)
        acc -= static_cast<const double*>(c)[(long long)s * cstride + j] * static_cast<const double*>(V)[j * ldv + i];
      static_cast<double*>(x)[i] = acc;
    }
  }
}

void launch_seg_multi_axpy(bool cplx, void* x, const void* V, long long ldv, int nv, const void* c, int cstride,
                           const long long* seg, int nseg, cudaStream_t s) {
  if (nv <= 0 || nseg <= 0) return;
  if (cplx) seg_multi_axpy_kernel<true><<<nseg, 256, 0, s>>>(x, V, ldv, nv, c, cstride, seg);
  else seg_multi_axpy_kernel<false><<<nseg, 256, 0, s>>>(x, V, ldv, nv, c, cstride, seg);
}

// x *= f(scal[s * sstride]) on segment s: f = 1/v (inv) or v
template <bool CPLX>
__global__ void __launch_bounds__(256) seg_scale_kernel(void* x, const double* scal, int sstride, int inv,
                                                        const long long* seg) {
  const int s = blockIdx.x;
  const long long lo = seg[s], hi = seg[s + 1];
  const double v = scal[(long long)s * sstride];
  const double f = inv ? 1.0 / v : v;
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    if (CPLX) { double2 a = static_cast<double2*>(x)[i]; a.x *= f; a.y *= f; static_cast<double2*>(x)[i] = a; }
    else static_cast<double*>(x)[i] *= f;
  }
}

void launch_seg_scale(bool cplx, void* x, const double* scal, int sstride, int inv, const long long* seg, int nseg,
                      cudaStream_t s) {
  if (nseg <= 0) return;
  if (cplx) seg_scale_kernel<true><<<nseg, 256, 0, s>>>(x, scal, sstride, inv, seg);
  else seg_scale_kernel<false><<<nseg, 256, 0, s>>>(x, scal, sstride, inv, seg);
}

// y = sum_j c[s * cstride + j] V_j on the segments with mask[s] != 0
template <bool CPLX>
__global__ void __launch_bounds__(256) seg_lincomb_kernel(void* y, const void* V, long long ldv, int nv,
                                                          const double* c, int cstride, const int* mask,
                                                          const long long* seg) {
  const int s = blockIdx.x;
  if (!mask[s]) return;
  const long long lo = seg[s], hi = seg[s + 1];
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    if (CPLX) {
      double2 acc = make_double2(0.0, 0.0);
      for (int j = 0; j < nv; ++j) {
        const double cj = c[(long long)s * cstride + j];
        const double2 v = static_cast<const double2*>(V)[j * ldv + i];
        acc.x += cj * v.x;
        acc.y += cj * v.y;
      }
      static_cast<double2*>(y)[i] = acc;
    } else {
      double acc = 0.0;
      for (int j = 0; j < nv; ++j) acc += c[(long long)s * cstride + j] * static_cast<const double*>(V)[j * ldv + i];
      static_cast<double*>(y)[i] = acc;
    }
  }
}

void launch_seg_lincomb(bool cplx, void* y, const void* V, long long ldv, int nv, const double* c, int cstride,
                        const int* mask, const long long* seg, int nseg, cudaStream_t s) {
  if (nseg <= 0) return;
  if (cplx) seg_lincomb_kernel<true><<<nseg, 256, 0, s>>>(y, V, ldv, nv, c, cstride, mask, seg);
  else seg_lincomb_kernel<false><<<nseg, 256, 0, s>>>(y, V, ldv, nv, c, cstride, mask, seg);
}

// per segment s: op 0: coef[2s] = beta_prev[s * bstride], coef[2s + 1] = Re(dot[s])
//                op 1: out[s * ostride] = sqrt(|Re(dot[s])|)
template <bool CPLX>
__global__ void seg_lanczos_scalar_kernel(int op, const void* dot, const double* beta_prev, int bstride, void* out,
                                          int ostride, int nseg) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  const double re = CPLX ? static_cast<const double2*>(dot)[s].x : static_cast<const double*>(dot)[s];
  if (op == 0) {
    const double b = beta_prev[(long long)s * bstride];
    if (CPLX) {
      static_cast<double2*>(out)[2 * s] = make_double2(b, 0.0);
      static_cast<double2*>(out)[2 * s + 1] = make_double2(re, 0.0);
    } else {
      static_cast<double*>(out)[2 * s] = b;
      static_cast<double*>(out)[2 * s + 1] = re;
    }
  } else {
    static_cast<double*>(out)[(long long)s * ostride] = sqrt(fabs(re));
  }
}

void launch_seg_lanczos_scalar(bool cplx, int op, const void* dot, const double* beta_prev, int bstride, void* out,
                               int ostride, int nseg, cudaStream_t s) {
  if (nseg <= 0) return;
  const int blocks = (nseg + 127) / 128;
  if (cplx) seg_lanczos_scalar_kernel<true><<<blocks, 128, 0, s>>>(op, dot, beta_prev, bstride, out, ostride, nseg);
  else seg_lanczos_scalar_kernel<false><<<blocks, 128, 0, s>>>(op, dot, beta_prev, bstride, out, ostride, nseg);
}

}  // namespace sadmrg
