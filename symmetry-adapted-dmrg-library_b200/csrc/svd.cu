// svd.cu -- one-sided (Hestenes) block Jacobi SVD of the psi sector blocks.
//
// Replaces the per-sector LAPACK gesvd of the reference
// (src/dense_inst.cpp:447-541, called from src/block_tensor_inst.cpp:535-557).
// Method: Hestenes one-sided Jacobi (Hestenes 1958; Demmel & Veselic 1992,
// with the parallel block ordering of Brent & Luk).  The C = min(m,n) columns
// of W (A, or A^H when m < n) are split into column blocks of b <= 16.  Every
// round of a sweep pairs the blocks by the circle method; one CTA loads the
// 2b columns of its pair into shared memory, runs one cyclic sweep of scalar
// rotations over all of their column pairs (one warp per pair), writes them
// back, and applies the accumulated 2b x 2b rotation to the matching columns
// of V.  Sweeps repeat until a full sweep performs no rotation, so the result
// keeps the high relative accuracy of one-sided Jacobi on small singular
// values, which the reference's 1e-10 relative cut-off depends on.
#include <cuda_runtime.h>
#include <cmath>
#include <vector>

#include "common.hpp"
#include "kernels.cuh"

namespace sadmrg {

constexpr int kSvdThreads = 512;
constexpr int kSvdWarps = kSvdThreads / 32;
constexpr size_t kSvdSmemBudget = 200 * 1024;

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

// One visit of a column-block pair: load its 2b columns into shared memory, one
// cyclic sweep of scalar rotations over all their column pairs, write back, and
// apply the accumulated rotation to the same columns of V.  Adds the number of
// rotations to *rotations.  Every thread of the block calls it.
template <bool CPLX>
__device__ void jacobi_pair_visit(const SvdJob& J, const SvdPair& P, void* work, void* vmat, double tol,
                                  unsigned char* smem_raw, int* rotations) {
  using T = typename SvdT<CPLX>::T;
  const int R = J.trans ? J.n : J.m;
  const int C = J.trans ? J.m : J.n;
  int cols[32];
  int nc = 0;
  for (int c = P.bi * P.b; c < min((P.bi + 1) * P.b, C); ++c) cols[nc++] = c;
  if (P.bj >= 0)
    for (int c = P.bj * P.b; c < min((P.bj + 1) * P.b, C); ++c) cols[nc++] = c;
  T* Ws = reinterpret_cast<T*>(smem_raw);                 // nc columns of R
  T* Q = Ws + (size_t)nc * R;                              // nc x nc
  __shared__ int local_rot;
  T* W = static_cast<T*>(work) + J.woff;
  T* V = static_cast<T*>(vmat) + J.voff;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) local_rot = 0;
  for (int e = tid; e < nc * R; e += kSvdThreads) {
    const int c = e / R, r = e % R;
    Ws[e] = W[r + (long long)cols[c] * R];
  }
  for (int e = tid; e < nc * nc; e += kSvdThreads) {
    if (CPLX) reinterpret_cast<double2*>(Q)[e] = make_double2((e % nc) == (e / nc) ? 1.0 : 0.0, 0.0);
    else reinterpret_cast<double*>(Q)[e] = (e % nc) == (e / nc) ? 1.0 : 0.0;
  }
  __syncthreads();
  const int N = nc + (nc & 1);
  for (int rnd = 0; rnd < N - 1; ++rnd) {
    for (int pi = warp; pi < N / 2; pi += kSvdWarps) {
      int p, q;
      if (pi == 0) { p = N - 1; q = rnd; }
      else { p = (rnd + pi) % (N - 1); q = (rnd - pi + (N - 1)) % (N - 1); }
      if (p >= nc || q >= nc) continue;
      if (p > q) { const int tmp = p; p = q; q = tmp; }
      T* wp = Ws + (size_t)p * R;
      T* wq = Ws + (size_t)q * R;
      double a = 0.0, b = 0.0, gr = 0.0, gi = 0.0;
      for (int r = lane; r < R; r += 32) {
        if (CPLX) {
          const double2 x = reinterpret_cast<double2*>(wp)[r], y = reinterpret_cast<double2*>(wq)[r];
          a += x.x * x.x + x.y * x.y;
          b += y.x * y.x + y.y * y.y;
          gr += x.x * y.x + x.y * y.y;
          gi += x.x * y.y - x.y * y.x;
        } else {
          const double x = reinterpret_cast<double*>(wp)[r], y = reinterpret_cast<double*>(wq)[r];
          a += x * x;
          b += y * y;
          gr += x * y;
        }
      }
      a = wsum(a);
      b = wsum(b);
      gr = wsum(gr);
      if (CPLX) gi = wsum(gi);
      const double g = CPLX ? sqrt(gr * gr + gi * gi) : fabs(gr);
      const double nrm = sqrt(a) * sqrt(b);
      if (!(nrm > 1e-300) || g <= tol * nrm) continue;
      // rotation zeroing the (p,q) entry of the 2x2 Gram matrix [[a, g],[g*, b]];
      // for |zeta| > 1e150, zeta^2 would overflow: t = 1 / (2 zeta) to double
      // precision there, and a t that underflows to 0 means the pair is already
      // orthogonal to working precision (no rotation, none counted)
      const double zeta = (b - a) / (2.0 * g);
      const double t = fabs(zeta) > 1e150 ? 0.5 / zeta
                                          : (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
      if (!(t != 0.0)) continue;
      const double c = 1.0 / sqrt(1.0 + t * t);
      const double s = c * t;
      // phase e^{i phi} = gamma / |gamma|
      const double er = CPLX ? gr / g : (gr >= 0.0 ? 1.0 : -1.0);
      const double ei = CPLX ? gi / g : 0.0;
      // [wp wq] <- [wp wq] [[c, s e^{i phi}], [-s e^{-i phi}, c]]
      for (int r = lane; r < R; r += 32) {
        if (CPLX) {
          const double2 x = reinterpret_cast<double2*>(wp)[r], y = reinterpret_cast<double2*>(wq)[r];
          // -s e^{-i phi} * y
          const double2 yp = make_double2(-s * (er * y.x + ei * y.y), -s * (er * y.y - ei * y.x));
          // s e^{i phi} * x
          const double2 xp = make_double2(s * (er * x.x - ei * x.y), s * (er * x.y + ei * x.x));
          reinterpret_cast<double2*>(wp)[r] = make_double2(c * x.x + yp.x, c * x.y + yp.y);
          reinterpret_cast<double2*>(wq)[r] = make_double2(xp.x + c * y.x, xp.y + c * y.y);
        } else {
          const double x = reinterpret_cast<double*>(wp)[r], y = reinterpret_cast<double*>(wq)[r];
          const double sg = s * er;
          reinterpret_cast<double*>(wp)[r] = c * x - sg * y;
          reinterpret_cast<double*>(wq)[r] = sg * x + c * y;
        }
      }
      for (int r = lane; r < nc; r += 32) {
        T* qp = Q + (size_t)p * nc;
        T* qq = Q + (size_t)q * nc;
        if (CPLX) {
          const double2 x = reinterpret_cast<double2*>(qp)[r], y = reinterpret_cast<double2*>(qq)[r];
          const double2 yp = make_double2(-s * (er * y.x + ei * y.y), -s * (er * y.y - ei * y.x));
          const double2 xp = make_double2(s * (er * x.x - ei * x.y), s * (er * x.y + ei * x.x));
          reinterpret_cast<double2*>(qp)[r] = make_double2(c * x.x + yp.x, c * x.y + yp.y);
          reinterpret_cast<double2*>(qq)[r] = make_double2(xp.x + c * y.x, xp.y + c * y.y);
        } else {
          const double x = reinterpret_cast<double*>(qp)[r], y = reinterpret_cast<double*>(qq)[r];
          const double sg = s * er;
          reinterpret_cast<double*>(qp)[r] = c * x - sg * y;
          reinterpret_cast<double*>(qq)[r] = sg * x + c * y;
        }
      }
      if (lane == 0) atomicAdd(&local_rot, 1);
    }
    __syncthreads();
  }
  const int nrot = local_rot;
  __syncthreads();
  if (nrot == 0) return;        // nothing moved: W and V stay as they are
  for (int e = tid; e < nc * R; e += kSvdThreads) {
    const int c = e / R, r = e % R;
    W[r + (long long)cols[c] * R] = Ws[e];
  }
  __syncthreads();
  // V[:, cols] <- V[:, cols] * Q, staged through the (now free) column area in row chunks
  const int chunk = max(1, min(C, (int)(((size_t)nc * R) / (size_t)max(nc, 1))));
  T* Vs = Ws;
  for (int r0 = 0; r0 < C; r0 += chunk) {
    const int rows = min(chunk, C - r0);
    for (int e = tid; e < rows * nc; e += kSvdThreads) {
      const int c = e / rows, r = e % rows;
      Vs[e] = V[(r0 + r) + (long long)cols[c] * C];
    }
    __syncthreads();
    for (int e = tid; e < rows * nc; e += kSvdThreads) {
      const int c = e / rows, r = e % rows;
      if (CPLX) {
        double sr = 0.0, si = 0.0;
        for (int k = 0; k < nc; ++k) {
          const double2 v = reinterpret_cast<double2*>(Vs)[r + k * rows];
          const double2 q = reinterpret_cast<double2*>(Q)[k + c * nc];
          sr += v.x * q.x - v.y * q.y;
          si += v.x * q.y + v.y * q.x;
        }
        reinterpret_cast<double2*>(V)[(r0 + r) + (long long)cols[c] * C] = make_double2(sr, si);
      } else {
        double sr = 0.0;
        for (int k = 0; k < nc; ++k)
          sr += reinterpret_cast<double*>(Vs)[r + k * rows] * reinterpret_cast<double*>(Q)[k + c * nc];
        reinterpret_cast<double*>(V)[(r0 + r) + (long long)cols[c] * C] = sr;
      }
    }
    __syncthreads();
  }
  if (tid == 0) atomicAdd(rotations, nrot);
}

template <bool CPLX>
__global__ void __launch_bounds__(kSvdThreads) jacobi_pair_kernel(const SvdJob* __restrict__ jobs,
                                                                  const SvdPair* __restrict__ pairs, void* work,
                                                                  void* vmat, double tol, int* rotations) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const SvdPair P = pairs[blockIdx.x];
  const SvdJob J = jobs[P.job];
  jacobi_pair_visit<CPLX>(J, P, work, vmat, tol, smem_raw, rotations);
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

template <bool CPLX>
__global__ void __launch_bounds__(kSvdThreads) jacobi_coop_kernel(const SvdJob* __restrict__ jobs, int nj,
                                                                  const SvdPair* __restrict__ pairs,
                                                                  const int* __restrict__ roff, int max_rounds,
                                                                  void* work, void* vmat, double tol, int* cnt,
                                                                  SvdCtl* ctl, int max_sweeps) {
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
    for (int r = 0; r < max_rounds; ++r) {
      for (int p = roff[r] + blockIdx.x; p < roff[r + 1]; p += gridDim.x) {
        const SvdPair P = pairs[p];
        if (done[P.job]) continue;
        const SvdJob J = jobs[P.job];
        jacobi_pair_visit<CPLX>(J, P, work, vmat, tol, smem_raw, cur + P.job);
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
__global__ void jacobi_init_kernel(const SvdJob* jobs, const void* a, void* work, void* vmat) {
  using T = typename SvdT<CPLX>::T;
  const SvdJob J = jobs[blockIdx.x];
  const int R = J.trans ? J.n : J.m, C = J.trans ? J.m : J.n;
  const T* A = static_cast<const T*>(a) + J.aoff;
  T* W = static_cast<T*>(work) + J.woff;
  T* V = static_cast<T*>(vmat) + J.voff;
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

static int pick_block(bool cplx, int R) {
  const size_t es = cplx ? 16 : 8;
  for (int b = 16; b >= 1; b /= 2) {
    const size_t need = ((size_t)2 * b * R + (size_t)4 * b * b) * es;
    if (need <= kSvdSmemBudget) return b;
  }
  return 0;
}

// Host driver.  Runs all sweeps in one cooperative launch when the device allows
// it, otherwise one launch per round and one host synchronisation per sweep to
// test convergence.  Returns the number of sweeps taken (or -1 when max_sweeps
// was reached).
int run_jacobi_svd(bool cplx, const void* a, void* work, void* vmat, double* sv, const std::vector<SvdJob>& hjobs,
                   int max_sweeps, cudaStream_t s, double* kernel_ms) {
  if (kernel_ms) *kernel_ms = -1.0;
  const int nj = (int)hjobs.size();
  if (nj == 0) return 0;
  std::vector<int> bsz(nj), nblk(nj), nrounds(nj);
  int max_rounds = 0, maxR = 0;
  size_t smem = 0;
  for (int j = 0; j < nj; ++j) {
    const int R = hjobs[j].trans ? hjobs[j].n : hjobs[j].m;
    const int C = hjobs[j].trans ? hjobs[j].m : hjobs[j].n;
    maxR = std::max(maxR, R);
    bsz[j] = pick_block(cplx, R);
    SADMRG_REQUIRE(bsz[j] > 0, SADMRG_ERR_LIMIT, "jacobi svd: sector block too tall for shared memory");
    nblk[j] = (C + bsz[j] - 1) / bsz[j];
    const int N = nblk[j] + (nblk[j] & 1);
    nrounds[j] = nblk[j] <= 1 ? 1 : N - 1;
    max_rounds = std::max(max_rounds, nrounds[j]);
    const int nc = std::min(C, 2 * bsz[j]);
    smem = std::max(smem, ((size_t)nc * R + (size_t)nc * nc) * (cplx ? 16 : 8));
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
  DevBuf djobs(sizeof(SvdJob) * nj, s), dpairs(sizeof(SvdPair) * flat.size(), s), dcnt(sizeof(int), s);
  SADMRG_CUDA(cudaMemcpyAsync(djobs.get(), hjobs.data(), sizeof(SvdJob) * nj, cudaMemcpyHostToDevice, s));
  SADMRG_CUDA(cudaMemcpyAsync(dpairs.get(), flat.data(), sizeof(SvdPair) * flat.size(), cudaMemcpyHostToDevice, s));
  dim3 ig(nj, 16);
  if (cplx) jacobi_init_kernel<true><<<ig, 256, 0, s>>>(djobs.as<SvdJob>(), a, work, vmat);
  else jacobi_init_kernel<false><<<ig, 256, 0, s>>>(djobs.as<SvdJob>(), a, work, vmat);
  SADMRG_CUDA(cudaGetLastError());
  if (cplx)
    SADMRG_CUDA(cudaFuncSetAttribute(jacobi_pair_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  else
    SADMRG_CUDA(cudaFuncSetAttribute(jacobi_pair_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const double tol = std::sqrt((double)std::max(maxR, 1)) * 2.220446049250313e-16;
  int sweeps = -1;
  int h_rot = 0;
  // preferred: every sweep in one cooperative launch (no host round trip per sweep)
  int dev = 0, coop = 0, nsm = 0, per_sm = 0;
  SADMRG_CUDA(cudaGetDevice(&dev));
  SADMRG_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  SADMRG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  if (cplx) {
    SADMRG_CUDA(cudaFuncSetAttribute(jacobi_coop_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SADMRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_coop_kernel<true>, kSvdThreads, smem));
  } else {
    SADMRG_CUDA(cudaFuncSetAttribute(jacobi_coop_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    SADMRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jacobi_coop_kernel<false>, kSvdThreads, smem));
  }
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
    void* args[] = {(void*)&pj, (void*)&njv, (void*)&pp, (void*)&pr, (void*)&mr, (void*)&a_work,
                    (void*)&a_vmat, (void*)&tolv, (void*)&pc, (void*)&pctl, (void*)&ms};
    if (cplx)
      SADMRG_CUDA(cudaLaunchCooperativeKernel((const void*)jacobi_coop_kernel<true>, dim3(grid), dim3(kSvdThreads),
                                              args, smem, s));
    else
      SADMRG_CUDA(cudaLaunchCooperativeKernel((const void*)jacobi_coop_kernel<false>, dim3(grid), dim3(kSvdThreads),
                                              args, smem, s));
    SvdCtl hctl{};
    SADMRG_CUDA(cudaMemcpyAsync(&hctl, dctl.get(), sizeof(SvdCtl), cudaMemcpyDeviceToHost, s));
    SADMRG_CUDA(cudaStreamSynchronize(s));
    SADMRG_REQUIRE(hctl.status == 0, SADMRG_ERR_CUDA, "jacobi svd: a grid barrier ran out of time");
    sweeps = hctl.sweeps;
    if (kernel_ms) *kernel_ms = (double)(hctl.t1 - hctl.t0) * 1e-6;
    if (cplx) jacobi_norms_kernel<true><<<nj, 256, 0, s>>>(djobs.as<SvdJob>(), work, sv);
    else jacobi_norms_kernel<false><<<nj, 256, 0, s>>>(djobs.as<SvdJob>(), work, sv);
    SADMRG_CUDA(cudaGetLastError());
    return sweeps;
  }
  for (int sw = 0; sw < max_sweeps; ++sw) {
    SADMRG_CUDA(cudaMemsetAsync(dcnt.get(), 0, sizeof(int), s));
    for (int r = 0; r < max_rounds; ++r) {
      const int np = roff[r + 1] - roff[r];
      if (np == 0) continue;
      if (cplx)
        jacobi_pair_kernel<true><<<np, kSvdThreads, smem, s>>>(djobs.as<SvdJob>(), dpairs.as<SvdPair>() + roff[r],
                                                               work, vmat, tol, dcnt.as<int>());
      else
        jacobi_pair_kernel<false><<<np, kSvdThreads, smem, s>>>(djobs.as<SvdJob>(), dpairs.as<SvdPair>() + roff[r],
                                                                work, vmat, tol, dcnt.as<int>());
    }
    SADMRG_CUDA(cudaGetLastError());
    SADMRG_CUDA(cudaMemcpyAsync(&h_rot, dcnt.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    SADMRG_CUDA(cudaStreamSynchronize(s));
    if (h_rot == 0) { sweeps = sw + 1; break; }
  }
  if (cplx) jacobi_norms_kernel<true><<<nj, 256, 0, s>>>(djobs.as<SvdJob>(), work, sv);
  else jacobi_norms_kernel<false><<<nj, 256, 0, s>>>(djobs.as<SvdJob>(), work, sv);
  SADMRG_CUDA(cudaGetLastError());
  return sweeps;
}

}  // namespace sadmrg
