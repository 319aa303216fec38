// batch.cpp -- many independent two-site problems solved together.
//
// Each instance is a frozen H_eff plan (one centre step of its own chain).  The
// plans are merged into one: instance i's psi / H psi segment starts at seg[i]
// of one long vector, its operators and stage-0 products at their own offsets of
// one operator buffer and one scratch buffer, so every batched matvec is one
// launch per stage for all instances (mma.sync for FP64, tcgen05 for 3xTF32).
// The Krylov recurrence runs segment-wise (one block per instance in every
// vector kernel), and the host keeps one tridiagonal problem per instance; the
// recurrence and its checks are those of lanczos1 (Lanczos::lanczos1,
// src/dmrg_inst.cpp:1286-1348), applied per instance.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "dmrg.hpp"

namespace sadmrg {

namespace {
template <class S> constexpr bool kCxB = ScalarInfo<S>::cplx;
}

template <class S>
void HeffBatch<S>::add(Ctx& c, const HeffPlan<S>& H) {
  SADMRG_REQUIRE(!ready, SADMRG_ERR_STATE, "batch: already finalized");
  Part p;
  p.job_terms = H.plan.job_terms;
  p.jobs = H.plan.jobs;
  p.job_stage = H.plan.job_stage;
  p.scratch = H.plan.scratch_elems;
  p.n = H.n;
  p.flops = H.flops;
  // The operators are copied on the batch's stream and the copy is awaited here:
  // the instance's buffers belong to its own handle (and stream), which the
  // caller may destroy as soon as this returns.
  const size_t bytes = H.opsbuf ? H.opsbuf->bytes() : 0;
  if (bytes) {
    p.ops = std::make_shared<DevBuf>(bytes, c.stream);
    SADMRG_CUDA(cudaMemcpyAsync(p.ops->get(), H.opsbuf->get(), bytes, cudaMemcpyDeviceToDevice, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  }
  parts.push_back(std::move(p));
}

template <class S>
void HeffBatch<S>::finalize(Ctx& c) {
  SADMRG_REQUIRE(!ready, SADMRG_ERR_STATE, "batch: already finalized");
  SADMRG_REQUIRE(!parts.empty(), SADMRG_ERR_STATE, "batch: no instances");
  const int np = (int)parts.size();
  seg.assign(np + 1, 0);
  std::vector<long long> ooff(np + 1, 0), xoff(np + 1, 0);
  for (int i = 0; i < np; ++i) {
    seg[i + 1] = seg[i] + parts[i].n;
    ooff[i + 1] = ooff[i] + (long long)(parts[i].ops ? parts[i].ops->bytes() / sizeof(S) : 0);
    xoff[i + 1] = xoff[i] + parts[i].scratch;
  }
  HeffPlan<S>& M = merged;
  M.n = seg[np];
  M.opsbuf = std::make_shared<DevBuf>(sizeof(S) * std::max<long long>(ooff[np], 1), c.stream);
  for (int i = 0; i < np; ++i)
    if (parts[i].ops && ooff[i + 1] > ooff[i])
      SADMRG_CUDA(cudaMemcpyAsync(M.opsbuf->template as<S>() + ooff[i], parts[i].ops->get(),
                                  sizeof(S) * (ooff[i + 1] - ooff[i]), cudaMemcpyDeviceToDevice, c.stream));
  GemmPlan& P = M.plan;
  for (int i = 0; i < np; ++i) {
    const Part& q = parts[i];
    auto base = [&](int buf) -> long long { return buf == 2 ? ooff[i] : buf == 3 ? xoff[i] : seg[i]; };
    for (size_t j = 0; j < q.jobs.size(); ++j) {
      const GemmJob& J = q.jobs[j];
      const int nj = P.add_job(q.job_stage[j], J.cbuf, J.coff + base(J.cbuf), J.m, J.n, J.ldc, J.flags);
      P.jobs[nj].tag = i;   // a masked matvec skips the jobs of converged instances
      for (const GemmTerm& t : q.job_terms[j])
        P.add_term(nj, t.abuf, t.aoff + base(t.abuf), t.lda, t.bbuf, t.boff + base(t.bbuf), t.ldb, t.k, t.flags,
                   t.ar, t.ai);
    }
    P.scratch_elems += q.scratch;
    M.flops += q.flops;
  }
  Bases cb{};
  cb.p[2] = M.opsbuf->get();
  P.finalize(c, kCxB<S>, /*mixed=*/true, &cb);
  M.scratch = std::make_shared<DevBuf>(sizeof(S) * std::max<long long>(P.scratch_elems, 1), c.stream);
  M.ntasks = (int)P.flat_terms.size();
  d_seg = std::make_shared<DevBuf>(sizeof(long long) * seg.size(), c.stream);
  SADMRG_CUDA(cudaMemcpyAsync(d_seg->get(), seg.data(), sizeof(long long) * seg.size(), cudaMemcpyHostToDevice,
                              c.stream));
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  parts.clear();   // the merged buffers hold everything now
  ready = true;
}

namespace {

// device and page-locked host work space of one batched Lanczos solve
template <class S>
struct BatchKrylov {
  Ctx& c;
  long long N;
  int ns, mlanc, bs;            // segments, Krylov size, beta row stride
  DevBuf ff, vh, dots, coef, beta, cdev, mask, norm, active;
  S* h_coef = nullptr;          // per step: coef (2 per segment) copied as it is made
  double* h_beta = nullptr;     // beta rows (ns x bs)
  S* h_dots = nullptr;          // 2 per segment
  double* h_cdev = nullptr;     // Ritz coefficients (ns x (mlanc + 1))
  int* h_mask = nullptr;
  int* h_active = nullptr;      // instances whose matvec work still runs (written only after a stream sync)
  BatchKrylov(Ctx& cc, long long n, int nseg, int ml) : c(cc), N(n), ns(nseg), mlanc(ml), bs(ml + 2) {
    ff.alloc(sizeof(S) * N * (mlanc + 1), c.stream);
    vh.alloc(sizeof(S) * N * 2, c.stream);
    dots.alloc(sizeof(S) * (size_t)ns * (mlanc + 2), c.stream);
    coef.alloc(sizeof(S) * (size_t)ns * 2, c.stream);
    beta.alloc(sizeof(double) * (size_t)ns * bs, c.stream);
    cdev.alloc(sizeof(double) * (size_t)ns * (mlanc + 1), c.stream);
    mask.alloc(sizeof(int) * ns, c.stream);
    norm.alloc(sizeof(double) * ns, c.stream);
    active.alloc(sizeof(int) * ns, c.stream);
    SADMRG_CUDA(cudaMemsetAsync(beta.get(), 0, sizeof(double) * (size_t)ns * bs, c.stream));
    SADMRG_CUDA(cudaMallocHost(&h_coef, sizeof(S) * (size_t)ns * 2 * (mlanc + 1)));
    SADMRG_CUDA(cudaMallocHost(&h_beta, sizeof(double) * (size_t)ns * bs));
    SADMRG_CUDA(cudaMallocHost(&h_dots, sizeof(S) * (size_t)ns * 2));
    SADMRG_CUDA(cudaMallocHost(&h_cdev, sizeof(double) * (size_t)ns * (mlanc + 1)));
    SADMRG_CUDA(cudaMallocHost(&h_mask, sizeof(int) * ns));
    SADMRG_CUDA(cudaMallocHost(&h_active, sizeof(int) * ns));
    std::fill(h_active, h_active + ns, 1);
    SADMRG_CUDA(cudaMemcpyAsync(active.get(), h_active, sizeof(int) * ns, cudaMemcpyHostToDevice, c.stream));
  }
  ~BatchKrylov() {
    cudaStreamSynchronize(c.stream);
    cudaFreeHost(h_coef);
    cudaFreeHost(h_beta);
    cudaFreeHost(h_dots);
    cudaFreeHost(h_cdev);
    cudaFreeHost(h_mask);
    cudaFreeHost(h_active);
  }
  S* F(int i) { return ff.as<S>() + (size_t)i * N; }
};

template <class S>
BatchStats batch_lanczos1(Ctx& c, const HeffBatch<S>& B, S* v, int mlanc, int prec) {
  constexpr bool CX = kCxB<S>;
  const HeffPlan<S>& H = B.merged;
  const int ns = B.nseg();
  const long long N = H.n;
  const long long* seg = B.d_seg->template as<long long>();
  BatchKrylov<S> K(c, N, ns, mlanc);
  const double tol = 1.e-6;
  BatchStats st;
  st.energy.assign(ns, 0.0);
  st.matvecs.assign(ns, 0);
  std::vector<char> done(ns, 0);
  std::vector<std::vector<double>> aal(ns, std::vector<double>(mlanc, 0.0)), nnl(ns, std::vector<double>(mlanc + 1, 0.0));
  // Converged instances are switched off in the matvec (their jobs skip all
  // work; their segments of the output keep stale values that nothing reads).
  auto matvec = [&](const S* in, S* out) {
    c.job_mask = K.active.template as<int>();
    try {
      H.apply(c, in, out, prec);
    } catch (...) {
      c.job_mask = nullptr;
      throw;
    }
    c.job_mask = nullptr;
    ++st.launches_matvec;
    for (int s = 0; s < ns; ++s)
      if (!done[s]) ++st.matvecs[s];
  };
  // x /= |x| on the masked segments (all when mask is null); norms below 1e-12 are left alone
  auto normalize = [&](S* x, bool masked) {
    launch_seg_multi_dot(CX, x, N, 1, x, seg, ns, K.dots.get(), c.stream);
    launch_seg_lanczos_scalar(CX, 1, K.dots.get(), nullptr, 0, K.norm.get(), 1, ns, c.stream);
    SADMRG_CUDA(cudaMemcpyAsync(K.h_beta, K.norm.get(), sizeof(double) * ns, cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    for (int s = 0; s < ns; ++s) {
      const double nr = K.h_beta[s];
      K.h_cdev[s] = (nr > 1e-12 && (!masked || K.h_mask[s])) ? 1.0 / nr : 1.0;
    }
    SADMRG_CUDA(cudaMemcpyAsync(K.norm.get(), K.h_cdev, sizeof(double) * ns, cudaMemcpyHostToDevice, c.stream));
    launch_seg_scale(CX, x, K.norm.template as<double>(), 1, 0, seg, ns, c.stream);
    c.launches += 4;
  };
  // Ritz vectors of the masked segments into v: coefficients in h_cdev (row stride mlanc + 1)
  auto ritz = [&](int nv) {
    SADMRG_CUDA(cudaMemcpyAsync(K.cdev.get(), K.h_cdev, sizeof(double) * (size_t)ns * (mlanc + 1),
                                cudaMemcpyHostToDevice, c.stream));
    SADMRG_CUDA(cudaMemcpyAsync(K.mask.get(), K.h_mask, sizeof(int) * ns, cudaMemcpyHostToDevice, c.stream));
    launch_seg_lincomb(CX, v, K.F(0), N, nv, K.cdev.template as<double>(), mlanc + 1, K.mask.template as<int>(), seg,
                       ns, c.stream);
    ++c.launches;
  };
  // Lanczos::check_eigenvector on the masked segments: normalise v, |<v|Hv>| / |Hv|
  std::vector<double> ov(ns, 0.0);
  auto check = [&]() {
    normalize(v, true);
    S* vv = K.vh.template as<S>();
    S* hv = vv + N;
    SADMRG_CUDA(cudaMemcpyAsync(vv, v, sizeof(S) * N, cudaMemcpyDeviceToDevice, c.stream));
    matvec(vv, hv);
    launch_seg_multi_dot(CX, vv, N, 2, hv, seg, ns, K.dots.get(), c.stream);
    ++c.launches;
    SADMRG_CUDA(cudaMemcpyAsync(K.h_dots, K.dots.get(), sizeof(S) * 2 * ns, cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    for (int s = 0; s < ns; ++s) {
      if (!K.h_mask[s]) continue;
      const double prod = std::sqrt(std::fabs(real_of(K.h_dots[2 * s + 1])));
      ov[s] = prod > 0 ? std::abs(K.h_dots[2 * s]) / prod : 0.0;
    }
  };
  auto tridiag = [&](int s, int m, std::vector<double>& eig, std::vector<double>& z) {
    eig.assign(aal[s].begin(), aal[s].begin() + m);
    std::vector<double> e(m, 0.0);
    for (int i = 0; i + 1 < m; ++i) e[i] = nnl[s][i + 1];
    tridiag_eig(m, eig, e, z);
  };

  // F(0) = normalised v
  SADMRG_CUDA(cudaMemcpyAsync(K.F(0), v, sizeof(S) * N, cudaMemcpyDeviceToDevice, c.stream));
  std::fill(K.h_mask, K.h_mask + ns, 1);
  normalize(K.F(0), false);

  int synced = 0;
  auto step = [&](int m) {
    matvec(K.F(m - 1), K.F(m));
    launch_seg_multi_dot(CX, K.F(m - 1), N, 1, K.F(m), seg, ns, K.dots.get(), c.stream);
    launch_seg_lanczos_scalar(CX, 0, K.dots.get(), K.beta.template as<double>() + (m - 1), K.bs, K.coef.get(), 0, ns,
                              c.stream);
    if (m >= 2)
      launch_seg_multi_axpy(CX, K.F(m), K.F(m - 2), N, 2, K.coef.get(), 2, seg, ns, c.stream);
    else
      launch_seg_multi_axpy(CX, K.F(m), K.F(m - 1), N, 1, K.coef.template as<S>() + 1, 2, seg, ns, c.stream);
    if (m >= 2) {
      launch_seg_multi_dot(CX, K.F(0), N, m, K.F(m), seg, ns, K.dots.get(), c.stream);
      launch_seg_multi_axpy(CX, K.F(m), K.F(0), N, m, K.dots.get(), m, seg, ns, c.stream);
    }
    launch_seg_multi_dot(CX, K.F(m), N, 1, K.F(m), seg, ns, K.dots.get(), c.stream);
    launch_seg_lanczos_scalar(CX, 1, K.dots.get(), nullptr, 0, K.beta.template as<double>() + m, K.bs, ns, c.stream);
    launch_seg_scale(CX, K.F(m), K.beta.template as<double>() + m, K.bs, 1, seg, ns, c.stream);
    c.launches += 9;
    SADMRG_CUDA(cudaMemcpyAsync(K.h_coef + (size_t)(m - 1) * 2 * ns, K.coef.get(), sizeof(S) * 2 * ns,
                                cudaMemcpyDeviceToHost, c.stream));
  };
  auto sync_to = [&](int m, std::vector<int>& brk) {
    SADMRG_CUDA(cudaMemcpyAsync(K.h_beta, K.beta.get(), sizeof(double) * (size_t)ns * K.bs, cudaMemcpyDeviceToHost,
                                c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    brk.assign(ns, 0);
    for (int s = 0; s < ns; ++s)
      for (int j = synced + 1; j <= m; ++j) {
        aal[s][j - 1] = real_of(K.h_coef[(size_t)(j - 1) * 2 * ns + 2 * s + 1]);
        nnl[s][j] = K.h_beta[(size_t)s * K.bs + j];
        if (!brk[s] && j >= 2 && nnl[s][j] < tol) brk[s] = j;
      }
    synced = m;
  };

  std::vector<double> eig, z;
  std::vector<int> brk;
  std::vector<double> e0(ns, 0.0);
  std::vector<int> finishing(ns, 0);
  step(1);
  if (mlanc > 2) {
    for (int m = 2; m < mlanc; ++m) {
      step(m);
      if (m % 4 != 0 && m != mlanc - 1) continue;
      sync_to(m, brk);
      bool any = false;
      std::fill(K.h_mask, K.h_mask + ns, 0);
      std::fill(K.h_cdev, K.h_cdev + (size_t)ns * (mlanc + 1), 0.0);
      for (int s = 0; s < ns; ++s) {
        finishing[s] = 0;
        if (done[s]) continue;
        const int mm = brk[s] ? brk[s] : m;
        if (!brk[s] && m % 4 != 0) continue;
        tridiag(s, mm, eig, z);
        e0[s] = eig[0];
        for (int j = 0; j < mm; ++j) K.h_cdev[(size_t)s * (mlanc + 1) + j] = z[j];
        K.h_mask[s] = 1;
        finishing[s] = brk[s] ? 1 : 0;
        any = true;
      }
      if (!any) continue;
      ritz(m + 1);
      check();
      bool all = true, changed = false;
      for (int s = 0; s < ns; ++s) {
        if (K.h_mask[s] && (finishing[s] || std::fabs(ov[s] - 1.0) < c.lanczos_ov_tol)) {
          done[s] = 1;
          st.energy[s] = e0[s];
          K.h_active[s] = 0;
          changed = true;
        }
        if (!done[s]) all = false;
      }
      if (all) return st;
      if (changed)   // check() synchronised the stream, so h_active is not being read by an earlier copy
        SADMRG_CUDA(cudaMemcpyAsync(K.active.get(), K.h_active, sizeof(int) * ns, cudaMemcpyHostToDevice, c.stream));
    }
  }
  // instances still open after mlanc - 1 steps: one more matvec, then the Ritz vector
  const int last = mlanc > 2 ? mlanc - 1 : 1;
  matvec(K.F(last), K.F(last + 1));
  launch_seg_multi_dot(CX, K.F(last), N, 1, K.F(last + 1), seg, ns, K.dots.get(), c.stream);
  ++c.launches;
  SADMRG_CUDA(cudaMemcpyAsync(K.h_dots, K.dots.get(), sizeof(S) * ns, cudaMemcpyDeviceToHost, c.stream));
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  std::fill(K.h_mask, K.h_mask + ns, 0);
  std::fill(K.h_cdev, K.h_cdev + (size_t)ns * (mlanc + 1), 0.0);
  for (int s = 0; s < ns; ++s) {
    if (done[s]) continue;
    aal[s][last] = real_of(K.h_dots[s]);
    tridiag(s, last + 1, eig, z);
    e0[s] = eig[0];
    for (int j = 0; j <= last; ++j) K.h_cdev[(size_t)s * (mlanc + 1) + j] = z[j];
    K.h_mask[s] = 1;
  }
  ritz(last + 1);
  check();
  for (int s = 0; s < ns; ++s)
    if (!done[s]) {
      done[s] = 1;
      st.energy[s] = e0[s];
    }
  return st;
}

}  // namespace

template <class S>
BatchStats batch_lanczos_solve(Ctx& c, const HeffBatch<S>& B, S* v, int mlanc, int prec) {
  SADMRG_REQUIRE(B.ready, SADMRG_ERR_STATE, "batch: not finalized");
  SADMRG_REQUIRE(mlanc >= 3, SADMRG_ERR_ARG, "batch lanczos: mlanc >= 3");
  if (prec == PREC_FP64) return batch_lanczos1<S>(c, B, v, mlanc, PREC_FP64);
  const double tol = c.lanczos_ov_tol;
  c.lanczos_ov_tol = std::max(tol, 1e-10);   // the split-precision phase stops no tighter (see lanczos_solve)
  BatchStats a;
  try {
    a = batch_lanczos1<S>(c, B, v, mlanc, prec);
  } catch (...) {
    c.lanczos_ov_tol = tol;
    throw;
  }
  c.lanczos_ov_tol = tol;
  BatchStats b = batch_lanczos1<S>(c, B, v, mlanc, PREC_FP64);   // FP64 restart
  for (size_t s = 0; s < b.matvecs.size(); ++s) b.matvecs[s] += a.matvecs[s];
  b.launches_matvec += a.launches_matvec;
  return b;
}

template struct HeffBatch<double>;
template struct HeffBatch<dcmplex>;
template BatchStats batch_lanczos_solve<double>(Ctx&, const HeffBatch<double>&, double*, int, int);
template BatchStats batch_lanczos_solve<dcmplex>(Ctx&, const HeffBatch<dcmplex>&, dcmplex*, int, int);

}  // namespace sadmrg
