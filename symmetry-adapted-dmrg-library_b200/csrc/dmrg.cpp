// dmrg.cpp -- H_eff plans, Lanczos, block SVD truncation and the sweep driver.
#include "dmrg.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>

namespace sadmrg {

template <class S> static constexpr bool kCx = ScalarInfo<S>::cplx;

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------------------
// Autotuner of the split-precision matvec.  Candidates: output tile width 64 or
// 128, times three ways to cut the reductions -- split-K chunks of at least 16 k
// slabs when the output tiles cannot fill the GPU, no split, or no item longer
// than 32 (or, at width 64, 16) slabs: the longest items set the time of a
// launch -- two CTAs per SM at width 64 (a 2-stage ring each, so one CTA's
// epilogue overlaps the other's MMAs), and, for the fastest of those, one
// cooperative launch for the whole matvec against one launch per stage.  Each candidate schedule is built on the plan itself and timed with
// CUDA events on the context's stream (one warm run, then the mean of three);
// the winner is cached per block-size histogram (GemmPlan::tune_key) for the
// life of the process, so later plans with the same histogram reuse it untimed.
// The FP64 path is not tuned: its schedule, and so its rounding, never depends
// on a timing.
namespace {
std::mutex g_tune_mu;
std::map<std::string, UmmaTune> g_tune_cache;
}

constexpr float kTuneMargin = 0.97f;

template <class S>
static void autotune_heff(Ctx& c, HeffPlan<S>& H) {
  GemmPlan& p = H.plan;
  if (p.umma && c.forced_tune.bn > 0) {
    p.tune = c.forced_tune;
    p.tune.source = 3;
    p.rebuild_umma(c, kCx<S>);
    return;
  }
  if (!p.umma || !c.autotune || c.fused_matvec >= 0 || c.prof) return;
  const std::string key = p.tune_key(kCx<S>);
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      const UmmaTune built = p.tune;
      const int built_bn = p.umma->bn;
      p.tune = it->second;
      p.tune.source = 2;
      if (p.tune.bn != built_bn || p.tune.kc_min != built.kc_min || p.tune.kc_max != built.kc_max ||
          p.tune.ctas != built.ctas)
        p.rebuild_umma(c, kCx<S>);
      return;
    }
  }
  const size_t nb = sizeof(S) * std::max<long long>(H.n, 1);
  DevBuf x(nb, c.stream), y(nb, c.stream);
  SADMRG_CUDA(cudaMemsetAsync(x.get(), 0, nb, c.stream));
  Bases b{};
  b.p[0] = x.get();
  b.p[1] = y.get();
  b.p[2] = H.opsbuf->get();
  b.p[3] = H.scratch->get();
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  UmmaTune win;
  float best = 1e30f;
  auto record = [&](float ms, const UmmaTune& t, int fused) {
    if (win.ncand >= 8) return;
    win.ms[win.ncand] = ms;
    win.cand_bn[win.ncand] = t.bn;
    win.cand_kc[win.ncand] = t.kc_min;
    win.cand_kmax[win.ncand] = t.kc_max;
    win.cand_fused[win.ncand] = fused;
    win.cand_ctas[win.ncand] = t.ctas;
    ++win.ncand;
  };
  try {
    SADMRG_CUDA(cudaEventCreate(&e0));
    SADMRG_CUDA(cudaEventCreate(&e1));
    auto time_current = [&]() -> float {
      p.run(c, kCx<S>, PREC_TF32X3, b);   // warm: first touch of the schedule
      SADMRG_CUDA(cudaEventRecord(e0, c.stream));
      for (int r = 0; r < 3; ++r) p.run(c, kCx<S>, PREC_TF32X3, b);
      SADMRG_CUDA(cudaEventRecord(e1, c.stream));
      SADMRG_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      SADMRG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      return ms / 3.f;
    };
    // {width, split floor, item cap, CTAs per SM}
    const int cands[7][4] = {{64, 16, 0, 1},  {128, 16, 0, 1}, {64, 0, 0, 1},  {128, 0, 0, 1},
                             {64, 16, 32, 1}, {64, 16, 0, 2},  {64, 16, 32, 2}};
    std::vector<std::tuple<int, size_t, size_t>> seen;   // schedules already timed: (bn, items, reductions)
    UmmaTune pick;
    for (const auto& cd : cands) {
      p.tune = UmmaTune{};
      p.tune.bn = cd[0];
      p.tune.kc_min = cd[1];
      p.tune.kc_max = cd[2];
      p.tune.ctas = cd[3];
      p.tune.fused = 0;
      if (!p.rebuild_umma(c, kCx<S>)) break;
      const auto fp = std::make_tuple(p.umma->bn * 4 + p.umma->ctas, p.umma->items.size(), p.umma->reds.size());
      if (std::find(seen.begin(), seen.end(), fp) != seen.end()) continue;   // the same schedule as one timed
      seen.push_back(fp);
      float ms = 0.f;
      try {
        ms = time_current();
      } catch (const Error&) {
        cudaGetLastError();   // a launch configuration this device refuses: not a candidate
        continue;
      }
      record(ms, p.tune, 0);
      // a later candidate must win by more than the timing noise (3%), so that
      // near-equal schedules resolve to the earlier one from run to run
      if (ms < best * kTuneMargin) { best = ms; pick = p.tune; }
    }
    // the fastest, also as one cooperative launch
    p.tune = pick;
    p.rebuild_umma(c, kCx<S>);
    p.tune.fused = 1;
    if (p.runs_fused(c, kCx<S>, PREC_TF32X3)) {
      try {
        const float ms = time_current();
        record(ms, pick, 1);
        if (ms < best * kTuneMargin) { best = ms; pick.fused = 1; }
      } catch (const Error&) {
        cudaGetLastError();
      }
    }
    win.bn = pick.bn;
    win.kc_min = pick.kc_min;
    win.kc_max = pick.kc_max;
    win.ctas = pick.ctas;
    win.fused = pick.fused;
  } catch (...) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  win.source = 1;
  p.tune = win;   // the schedule built last is win's (the fused run shares it)
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune_cache[key] = win;
}

// ---------------------------------------------------------------------------
// H_eff * psi plan (DMRG::hamiltonian_vector_multiplication_idmrg, src/dmrg_inst.cpp:283-371,
// and BlockTensor::hamiltonian_vector_multiplication, src/block_tensor_inst.cpp:2170-2318)
template <class S>
HeffPlan<S> build_heff(Ctx& c, const BTensor<S>& psi, const BTensor<S>* hhL, const BTensor<S>* hhR,
                       const std::vector<const BTensor<S>*>& opl, const std::vector<PairTerm>& terms, bool tune) {
  HeffPlan<S> H;
  H.psi_st = psi.st;
  H.psi_off = psi.off;
  H.n = psi.nelem;
  // pack every operator the plan reads into one buffer (base id 2)
  std::vector<long long> base(opl.size(), -1);
  long long tot = 0, hl = -1, hr = -1;
  if (hhL && !hhL->null()) { hl = tot; tot += hhL->nelem; }
  if (hhR && !hhR->null()) { hr = tot; tot += hhR->nelem; }
  for (size_t i = 0; i < opl.size(); ++i)
    if (opl[i] && !opl[i]->null()) { base[i] = tot; tot += opl[i]->nelem; }
  H.opsbuf = std::make_shared<DevBuf>(sizeof(S) * std::max<long long>(tot, 1), c.stream);
  auto cp = [&](const BTensor<S>* t, long long at) {
    if (t->nelem > 0)
      SADMRG_CUDA(cudaMemcpyAsync(H.opsbuf->template as<S>() + at, t->data(), sizeof(S) * t->nelem, cudaMemcpyDeviceToDevice,
                                  c.stream));
  };
  if (hl >= 0) cp(hhL, hl);
  if (hr >= 0) cp(hhR, hr);
  for (size_t i = 0; i < opl.size(); ++i)
    if (base[i] >= 0) cp(opl[i], base[i]);

  GemmPlan& p = H.plan;
  const Struct& ps0 = psi.st;
  auto same = [](const Bond& a, const Bond& b) { return a.q == b.q && a.d == b.d; };
  SADMRG_REQUIRE(ps0.nbond() == 2, SADMRG_ERR_ARG, "heff: psi must have two bonds");
  if (hl >= 0)
    SADMRG_REQUIRE(hhL->st.nbond() == 2 && same(hhL->st.bonds[0], ps0.bonds[0]) && same(hhL->st.bonds[1], ps0.bonds[0]),
                   SADMRG_ERR_ARG, "heff: left block Hamiltonian does not match psi");
  if (hr >= 0)
    SADMRG_REQUIRE(hhR->st.nbond() == 2 && same(hhR->st.bonds[0], ps0.bonds[1]) && same(hhR->st.bonds[1], ps0.bonds[1]),
                   SADMRG_ERR_ARG, "heff: right block Hamiltonian does not match psi");
  for (auto& t : terms) {
    const BTensor<S>* a = opl[t.op1];
    const BTensor<S>* b = opl[t.op2];
    if (!a || !b || a->null() || b->null()) continue;
    SADMRG_REQUIRE(a->st.nbond() == 3 && b->st.nbond() == 3 && same(a->st.bonds[0], ps0.bonds[0]) &&
                       same(a->st.bonds[2], ps0.bonds[0]) && same(b->st.bonds[0], ps0.bonds[1]) &&
                       same(b->st.bonds[2], ps0.bonds[1]) && a->st.bonds[1].q == b->st.bonds[1].q &&
                       a->st.bonds[1].d == b->st.bonds[1].d,
                   SADMRG_ERR_ARG, "heff: operator bonds do not match psi");
  }
  const std::vector<Blk> P = blocks_of(psi);
  std::vector<int> job_of(psi.nten(), -1);
  for (auto& b : P) job_of[b.idx] = p.add_job(1, 1, b.off, b.d[0], b.d[1], b.d[0], 0);
  const Struct& ps = psi.st;
  int q[8], d[8];
  // diagonal terms: hh_L^T psi  (contract(hh[il], 0, vec1, 0))
  if (hl >= 0) {
    const Bond& cb = hhL->st.bonds[0];
    for (auto& o : P) {
      for (int j = 0; j < cb.nmom(); ++j) {
        int qa[2] = {cb.q[j], o.q[0]};   // hh block (j, x)
        int qb[2] = {cb.q[j], o.q[1]};   // psi block (j, b)
        if (!hhL->st.allowed_labels(qa) || !ps.allowed_labels(qb)) continue;
        const long ka = hhL->st.index(qa), kb = ps.index(qb);
        if (ka < 0 || kb < 0 || !hhL->present(ka) || !psi.present(kb)) continue;
        p.add_term(job_of[o.idx], 2, hl + hhL->off[ka], cb.d[j], 0, psi.off[kb], cb.d[j], cb.d[j], TF_TA, 1.0, 0.0);
      }
    }
  }
  // diagonal terms: psi hh_R  (contract(vec1, 1, hh[ir], 0))
  if (hr >= 0) {
    const Bond& cb = hhR->st.bonds[0];
    for (auto& o : P) {
      for (int j = 0; j < cb.nmom(); ++j) {
        int qa[2] = {o.q[0], cb.q[j]};   // psi block (a, j)
        int qb[2] = {cb.q[j], o.q[1]};   // hh block (j, y)
        if (!ps.allowed_labels(qa) || !hhR->st.allowed_labels(qb)) continue;
        const long ka = ps.index(qa), kb = hhR->st.index(qb);
        if (ka < 0 || kb < 0 || !psi.present(ka) || !hhR->present(kb)) continue;
        p.add_term(job_of[o.idx], 0, psi.off[ka], o.d[0], 2, hr + hhR->off[kb], cb.d[j], cb.d[j], 0, 1.0, 0.0);
      }
    }
  }
  // pair terms: out(a',b') += fac * op1^T psi op2
  for (auto& t : terms) {
    const BTensor<S>& o1 = *opl[t.op1];
    const BTensor<S>& o2 = *opl[t.op2];
    if (o1.null() || o2.null()) continue;
    SADMRG_REQUIRE(o1.st.bonds[2].q == ps.bonds[0].q && o2.st.bonds[2].q == ps.bonds[1].q, SADMRG_ERR_ARG,
                   "heff: operator bonds do not match psi");
    const auto O1 = blocks_of(o1);
    std::vector<std::array<int, 3>> o2q;
    std::vector<long long> o2off;
    std::vector<int> o2d0;
    for (long l = 0; l < o2.nten(); ++l)
      if (o2.st.block(l, q, d) && o2.present(l)) {
        o2q.push_back({q[0], q[1], q[2]});
        o2off.push_back(base[t.op2] + o2.off[l]);
        o2d0.push_back(d[0] * d[1]);
      }
    for (auto& pk : P)
      for (auto& a : O1) {
        if (a.q[0] != pk.q[0]) continue;
        SADMRG_REQUIRE(a.d[1] == 1, SADMRG_ERR_ARG, "heff: channel leg dim != 1");
        int x = -1;
        long long xo = 0;
        for (size_t l = 0; l < o2q.size(); ++l) {
          if (o2q[l][0] != pk.q[1] || a.q[1] != o2q[l][1]) continue;
          int lab[2] = {a.q[2], o2q[l][2]};
          if (!ps.allowed_labels(lab)) continue;
          const long m = ps.index(lab);
          if (m < 0 || !psi.present(m)) continue;
          double fac = 1.0;
          if (c.sym == Sym::SU2) {
            fac = c.cgc->hamilt_vec(a.q[0], a.q[1], a.q[2]);
            if (std::fabs(fac) < 1e-12) continue;
          }
          if (x < 0) {
            xo = p.alloc_scratch((long long)a.d[2] * pk.d[1]);
            x = p.add_job(0, 3, xo, a.d[2], pk.d[1], a.d[2], 0);
            p.add_term(x, 2, base[t.op1] + a.off, a.d[0], 0, pk.off, pk.d[0], pk.d[0], TF_TA, 1.0, 0.0);
          }
          p.add_term(job_of[m], 3, xo, a.d[2], 2, o2off[l], o2d0[l], pk.d[1], 0, fac, 0.0);
        }
      }
  }
  Bases cb{};
  cb.p[2] = H.opsbuf->get();
  p.finalize(c, kCx<S>, /*mixed=*/true, &cb);
  H.scratch = std::make_shared<DevBuf>(sizeof(S) * std::max<long long>(p.scratch_elems, 1), c.stream);
  H.flops = p.flops;
  H.bytes = (2 * H.n + tot) * (long long)sizeof(S);
  H.ntasks = (int)p.flat_terms.size();
  if (tune || c.forced_tune.bn > 0) autotune_heff(c, H);
  return H;
}

template <class S>
void HeffPlan<S>::apply(Ctx& c, const S* psi, S* out, int prec) const {
  Bases b{};
  b.p[0] = const_cast<S*>(psi);
  b.p[1] = out;
  b.p[2] = opsbuf->get();
  b.p[3] = scratch->get();
  plan.run(c, kCx<S>, prec, b);
  penalty(c, psi, out);
}

template <class S>
void HeffPlan<S>::penalty(Ctx& c, const S* psi, S* out) const {
  if (npen <= 0) return;
  launch_multi_dot(kCx<S>, pen_o->get(), n, npen, psi, n, c.d_partial, c.npart, pen_dot->get(), c.d_counter,
                   c.stream);
  launch_multi_axpy(kCx<S>, out, pen_wo->get(), n, npen, pen_dot->get(), n, c.stream);
  c.launches += 3;
}

// ---------------------------------------------------------------------------
// symmetric tridiagonal eigenproblem (replaces LAPACK dstev, src/dmrg_inst.cpp:1216-1231):
// implicit QL with Wilkinson-type shifts (the tql2 algorithm of Bowdler, Martin,
// Reinsch and Wilkinson, 1968).  d: diagonal, e[i]: coupling of i and i+1.
// On return d is ascending and z (column-major n x n) holds the eigenvectors.
void tridiag_eig(int n, std::vector<double>& d, std::vector<double> e, std::vector<double>& z) {
  z.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) z[i + (size_t)i * n] = 1.0;
  e.resize(n, 0.0);
  if (n > 0) e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0, m;
    do {
      for (m = l; m < n - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= 2.220446049250313e-16 * dd) break;
      }
      if (m != l) {
        if (iter++ == 100) throw Error(SADMRG_ERR_NUMERIC, "tridiagonal QL did not converge");
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? std::fabs(r) : -std::fabs(r)));
        double s = 1.0, cc = 1.0, pp = 0.0;
        int i;
        bool deflated = false;
        for (i = m - 1; i >= l; --i) {
          double f = s * e[i], b = cc * e[i];
          e[i + 1] = (r = std::hypot(f, g));
          if (r == 0.0) { d[i + 1] -= pp; e[m] = 0.0; deflated = true; break; }
          s = f / r;
          cc = g / r;
          g = d[i + 1] - pp;
          r = (d[i] - g) * s + 2.0 * cc * b;
          d[i + 1] = g + (pp = s * r);
          g = cc * r - b;
          for (int k = 0; k < n; ++k) {
            f = z[k + (size_t)(i + 1) * n];
            z[k + (size_t)(i + 1) * n] = s * z[k + (size_t)i * n] + cc * f;
            z[k + (size_t)i * n] = cc * z[k + (size_t)i * n] - s * f;
          }
        }
        if (deflated) continue;
        d[l] -= pp;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return d[a] < d[b]; });
  std::vector<double> d2(n), z2((size_t)n * n);
  for (int k = 0; k < n; ++k) {
    d2[k] = d[ord[k]];
    std::memcpy(&z2[(size_t)k * n], &z[(size_t)ord[k] * n], sizeof(double) * n);
  }
  d.swap(d2);
  z.swap(z2);
}

// ---------------------------------------------------------------------------
// Lanczos
template <class S>
struct Krylov {
  Ctx& c;
  long long n;
  int mlanc;
  DevBuf ff, vh, coef, dots, beta, cdev;
  Krylov(Ctx& cc, long long nn, int ml) : c(cc), n(nn), mlanc(ml) {
    ff.alloc(sizeof(S) * n * (mlanc + 1), c.stream);
    vh.alloc(sizeof(S) * n * 2, c.stream);
    coef.alloc(sizeof(S) * (mlanc + 4), c.stream);
    dots.alloc(sizeof(S) * (mlanc + 4), c.stream);
    beta.alloc(sizeof(double) * (mlanc + 4), c.stream);
    cdev.alloc(sizeof(double) * (mlanc + 4), c.stream);
    SADMRG_CUDA(cudaMemsetAsync(beta.get(), 0, sizeof(double) * (mlanc + 4), c.stream));
  }
  S* F(int i) { return ff.as<S>() + (size_t)i * n; }
  void mdot(const S* V, int nv, const S* x, void* out, int scalar_op = -1, const double* beta_prev = nullptr,
            void* scalar_out = nullptr) {
    launch_multi_dot(kCx<S>, V, n, nv, x, n, c.d_partial, c.npart, out, c.d_counter, c.stream, scalar_op, beta_prev,
                     scalar_out);
    ++c.launches;
  }
  S dot_host(const S* a, const S* b) {  // <a|b>
    mdot(a, 1, b, dots.get());
    S r;
    SADMRG_CUDA(cudaMemcpyAsync(&r, dots.get(), sizeof(S), cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    return r;
  }
  void scale_host(S* x, double s) {
    launch_scale(kCx<S>, x, s, 0.0, n, c.stream);
    ++c.launches;
  }
  // vout = sum_j coef[j] F(j)
  void ritz(S* vout, const std::vector<double>& z, int m) {
    SADMRG_CUDA(cudaMemcpyAsync(cdev.get(), z.data(), sizeof(double) * m, cudaMemcpyHostToDevice, c.stream));
    launch_lincomb(kCx<S>, vout, F(0), n, m, cdev.as<double>(), n, c.stream);
    ++c.launches;
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  }
};

template <class S>
LanczosStats lanczos1(Ctx& c, const HeffPlan<S>& H, S* v, int mlanc, int prec, bool residual_test,
                      int check_every, bool variant2) {
  if (!residual_test || check_every < 1) check_every = 4;
  if (variant2) check_every = mlanc + 1;   // lanczos2: no check points before the last step
  LanczosStats st;
  const long long n = H.n;
  Krylov<S> K(c, n, mlanc);
  std::vector<double> aal(mlanc, 0.0), nnl(mlanc + 1, 0.0), eig, z;
  const double tol = 1.e-6;
  auto matvec = [&](const S* in, S* out) {
    H.apply(c, in, out, prec);
    ++st.matvecs;
    if (prec == PREC_FP64) ++st.matvecs_fp64;
  };
  auto diatridiag = [&](int m) {
    eig.assign(aal.begin(), aal.begin() + m);
    std::vector<double> e(m, 0.0);
    for (int i = 0; i + 1 < m; ++i) e[i] = nnl[i + 1];
    tridiag_eig(m, eig, e, z);
  };
  auto ritz_vec = [&](int m) {
    std::vector<double> col(z.begin(), z.begin() + m);  // eigenvector of the lowest Ritz value
    K.ritz(v, col, m);
  };
  // Lanczos::check_eigenvector (src/dmrg_inst.cpp:1241-1254)
  auto check = [&](double& ee, double& ov) {
    S* vv = K.vh.template as<S>();
    S* hv = vv + n;
    const double nor = std::sqrt(std::fabs(real_of(K.dot_host(v, v))));
    K.scale_host(v, 1.0 / nor);
    SADMRG_CUDA(cudaMemcpyAsync(vv, v, sizeof(S) * n, cudaMemcpyDeviceToDevice, c.stream));
    matvec(vv, hv);
    K.mdot(vv, 2, hv, K.dots.get());  // <v|h>, <h|h>
    S r[2];
    SADMRG_CUDA(cudaMemcpyAsync(r, K.dots.get(), sizeof(S) * 2, cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    const double prod = std::sqrt(std::fabs(real_of(r[1])));
    ee = prod;
    ov = std::abs(r[0]) / prod;
    st.overlap = ov;
  };
  // ff[0] = normalised v (Lanczos::initialize_lanczos, src/dmrg_inst.cpp:1201-1213)
  SADMRG_CUDA(cudaMemcpyAsync(K.F(0), v, sizeof(S) * n, cudaMemcpyDeviceToDevice, c.stream));
  {
    const double nor = std::sqrt(std::fabs(real_of(K.dot_host(K.F(0), K.F(0)))));
    if (nor > 1e-12) K.scale_host(K.F(0), 1.0 / nor);
  }
  // one Lanczos step: F(m) = H F(m-1) - a F(m-1) - b F(m-2), reorthogonalised, normalised.
  // a and b go to page-locked host memory without a synchronisation; the host reads
  // them at the next check point (every 4 steps, as the reference checks), so the
  // steps in between queue back to back on the stream.
  const int pin_stride = kCx<S> ? 2 : 1;
  SADMRG_REQUIRE((mlanc + 2) * (pin_stride + 1) <= Ctx::kPinnedDoubles, SADMRG_ERR_LIMIT,
                 "lanczos: mlanc too large for the pinned scalar buffer");
  double* pin_a = c.h_pinned;                             // Re(a_m) at pin_a[(m-1)*stride]
  double* pin_b = c.h_pinned + (mlanc + 2) * pin_stride;  // b_m
  int synced = 0;                                          // steps whose a, b are on the host
  auto step = [&](int m, bool reorth) {
    matvec(K.F(m - 1), K.F(m));
    K.mdot(K.F(m - 1), 1, K.F(m), K.dots.get(), 0, K.beta.template as<double>() + (m - 1), K.coef.get());
    if (m >= 2)
      launch_multi_axpy(kCx<S>, K.F(m), K.F(m - 2), n, 2, K.coef.get(), n, c.stream);
    else
      launch_multi_axpy(kCx<S>, K.F(m), K.F(m - 1), n, 1, K.coef.template as<S>() + 1, n, c.stream);
    ++c.launches;
    if (reorth) {
      K.mdot(K.F(0), m, K.F(m), K.dots.get());
      launch_multi_axpy(kCx<S>, K.F(m), K.F(0), n, m, K.dots.get(), n, c.stream);
      ++c.launches;
    }
    K.mdot(K.F(m), 1, K.F(m), K.dots.get(), 1, nullptr, K.beta.template as<double>() + m);
    launch_scale_inv(kCx<S>, K.F(m), K.beta.template as<double>() + m, n, c.stream);
    ++c.launches;
    SADMRG_CUDA(cudaMemcpyAsync(pin_a + (m - 1) * pin_stride, K.coef.template as<S>() + 1, sizeof(S),
                                cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaMemcpyAsync(pin_b + m, K.beta.template as<double>() + m, sizeof(double), cudaMemcpyDeviceToHost,
                                c.stream));
    st.iters = m;
  };
  // bring a, b of steps (synced, m] to the host; returns the first step in that
  // range whose b broke down (< tol), or 0.  Like the reference, the test starts
  // at step 2 (step 1's b is never tested, src/dmrg_inst.cpp:1296-1326).
  auto sync_to = [&](int m) -> int {
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    int brk = 0;
    for (int j = synced + 1; j <= m; ++j) {
      aal[j - 1] = pin_a[(j - 1) * pin_stride];
      nnl[j] = pin_b[j];
      if (!brk && j >= 2 && nnl[j] < tol) brk = j;
    }
    synced = m;
    return brk;
  };
  double ee = 0.0, ov = 0.0;
  step(1, false);
  if (mlanc == 2) {
    sync_to(1);
    if (nnl[1] < tol) {
      diatridiag(1);
      ritz_vec(1);
      st.energy = eig[0];
      return st;
    }
    matvec(K.F(1), K.F(2));
    const S a1 = K.dot_host(K.F(1), K.F(2));
    aal[1] = real_of(a1);
    diatridiag(2);
    ritz_vec(2);
    st.energy = eig[0];
    return st;
  }
  // The reference tests b < tol after every step and checks the eigenvector every
  // 4 steps (src/dmrg_inst.cpp:1313-1345); here both are evaluated at the check
  // points, and a breakdown found there is handled as if it had been seen at its
  // own step: the tridiagonal and the Ritz vector use the steps before it only,
  // and the steps queued after it are discarded.
  for (int m = 2; m < mlanc; ++m) {
    step(m, true);
    if (m % check_every != 0 && m != mlanc - 1) continue;
    const int brk = sync_to(m);
    if (brk && variant2) {
      // Lanczos::lanczos2 returns at a breakdown with the Ritz pair of the steps
      // before it (computed in its previous iteration; at step 2 that is T_1)
      st.iters = brk;
      diatridiag(brk - 1);
      ritz_vec(brk - 1);
      K.scale_host(v, 1.0 / std::sqrt(std::fabs(real_of(K.dot_host(v, v)))));
      st.energy = eig[0];
      return st;
    }
    if (brk) {
      st.iters = brk;
      diatridiag(brk);
      ritz_vec(brk);
      check(ee, ov);
      st.energy = eig[0];
      return st;
    }
    diatridiag(m);
    if (m % check_every == 0) {
      if (residual_test) {
        // |H y - theta y| = b_m |z_m| for the Ritz pair (theta, y) of the m steps; the
        // overlap test |<y|Hy>|/|Hy| - 1 ~ r^2 / (2 theta^2) without the check matvec
        const double r = nnl[m] * std::fabs(z[m - 1]);
        if (r * r < 2.0 * c.lanczos_ov_tol * eig[0] * eig[0]) {
          ritz_vec(m);
          st.energy = eig[0];
          st.overlap = 1.0 - r * r / (2.0 * eig[0] * eig[0]);
          return st;
        }
        continue;
      }
      ritz_vec(m);
      check(ee, ov);
      if (std::fabs(ov - 1.0) < c.lanczos_ov_tol) { st.energy = eig[0]; return st; }
    }
  }
  sync_to(mlanc - 1);
  matvec(K.F(mlanc - 1), K.F(mlanc));
  aal[mlanc - 1] = real_of(K.dot_host(K.F(mlanc - 1), K.F(mlanc)));
  diatridiag(mlanc);
  ritz_vec(mlanc);
  if (!variant2) check(ee, ov);
  st.energy = eig[0];
  return st;
}

template <class S>
LanczosStats lanczos2(Ctx& c, const HeffPlan<S>& H, S* v, int mlanc) {
  return lanczos1<S>(c, H, v, mlanc, PREC_FP64, false, 4, /*variant2=*/true);
}

template <class S>
LanczosStats lanczos_solve(Ctx& c, const HeffPlan<S>& H, S* v, int mlanc, int prec) {
  if (prec == PREC_FP64) return lanczos1<S>(c, H, v, mlanc, PREC_FP64);
  // Split-precision Krylov first.  Its stop test is held no tighter than 1e-10:
  // |<v|Hv>|/|Hv| - 1 ~ |error of v|^2, and the 3xTF32 operator (relative error
  // ~1e-7) leaves v accurate to ~1e-5 at best, so a tighter test only buys
  // matvecs the FP64 restart makes up for anyway.
  // It stops on the Lanczos residual estimate b_m |z_m| (no check matvecs); so
  // does the FP64 restart below (the reference's lanczos1 with FP64 matvecs,
  // tested after every step).  prec == PREC_FP64 alone keeps the reference's checks.
  const double tol = c.lanczos_ov_tol;
  c.lanczos_ov_tol = std::max(tol, 1e-10);
  LanczosStats a;
  try {
    a = lanczos1<S>(c, H, v, mlanc, prec, /*residual_test=*/true);
  } catch (...) {
    c.lanczos_ov_tol = tol;
    throw;
  }
  c.lanczos_ov_tol = tol;
  // FP64 defect-correction restart: from a vector already near the TF32 floor it
  // converges within a few steps, so it tests the (free) residual estimate after
  // every step rather than spending a check matvec every 4 steps
  LanczosStats b = lanczos1<S>(c, H, v, mlanc, PREC_FP64, /*residual_test=*/true, /*check_every=*/1);
  b.matvecs += a.matvecs;
  b.iters += a.iters;
  return b;
}

// ---------------------------------------------------------------------------
// block SVD and truncation (BlockTensor::svd, src/block_tensor_inst.cpp:501-637)
template <class S>
SvdStats block_svd(Ctx& c, const BTensor<S>& psi, BTensor<S>& tu, double p1, BTensor<S>& tv, double p2,
                   int max_dcut, std::vector<double>* wout) {
  SvdStats out;
  const Bond bb20 = tu.st.bonds[0], bb21 = tu.st.bonds[1], bb22 = tv.st.bonds[0], bb23 = tv.st.bonds[1];
  const Bond bb0 = Bond::fuse(c.sym, bb20, bb21), bb1 = Bond::fuse(c.sym, bb22, bb23);
  const int nm1 = bb0.nmom(), nm2 = bb1.nmom();
  SADMRG_REQUIRE(psi.st.nbond() == 2 && psi.st.bonds[0].q == bb0.q && psi.st.bonds[1].q == bb1.q &&
                     psi.st.bonds[0].d == bb0.d && psi.st.bonds[1].d == bb1.d,
                 SADMRG_ERR_ARG, "svd: psi does not match the fused bonds of the site tensors");
  std::vector<SvdJob> jobs;
  std::vector<int> job_of(nm1, -1), sec_j(nm1, -1);
  long long wtot = 0, stot = 0;
  for (int i = 0; i < nm1; ++i)
    for (int j = 0; j < nm2; ++j) {
      if (bb0.q[i] != bb1.q[j] || !psi.present(i + (long)j * nm1)) continue;
      SvdJob J{};
      J.m = bb0.d[i];
      J.n = bb1.d[j];
      J.trans = J.m < J.n ? 1 : 0;
      const long long R = std::max(J.m, J.n), C = std::min(J.m, J.n);
      J.aoff = psi.off[i + (long)j * nm1];
      J.woff = wtot;
      wtot += R * C;
      J.voff = wtot;
      wtot += C * C;
      J.soff = stot;
      stot += C;
      job_of[i] = (int)jobs.size();
      sec_j[i] = j;
      jobs.push_back(J);
    }
  DevBuf wv(sizeof(S) * std::max<long long>(wtot, 1), c.stream), sv(sizeof(double) * std::max<long long>(stot, 1), c.stream);
  const double tj = now_s();
  const int sweeps = run_jacobi_svd(kCx<S>, psi.data(), wv.get(), wv.get(), sv.as<double>(), jobs, 60, c.stream,
                                    &out.jacobi_kernel_ms, c.svd_qr, c.svd_stream, c.svd_block);
  out.jacobi_s = now_s() - tj;
  for (auto& J : jobs) {
    out.max_rows = std::max(out.max_rows, std::max(J.m, J.n));
    out.max_cols = std::max(out.max_cols, std::min(J.m, J.n));
  }
  c.launches += 1;
  SADMRG_REQUIRE(sweeps > 0 || jobs.empty(), SADMRG_ERR_NUMERIC, "svd: Jacobi sweeps did not converge");
  out.sweeps_max = sweeps;
  std::vector<double> hs(stot);
  if (stot > 0) SADMRG_CUDA(cudaMemcpyAsync(hs.data(), sv.get(), sizeof(double) * stot, cudaMemcpyDeviceToHost, c.stream));
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  // SADMRG_VERBOSE=2: every block's singular values (in the Jacobi's column order)
  if (const char* v = std::getenv("SADMRG_VERBOSE"); v && v[0] == '2')
    for (const SvdJob& J : jobs) {
      std::fprintf(stderr, "  block %dx%d:", J.m, J.n);
      for (int k = 0; k < std::min(J.m, J.n); ++k) std::fprintf(stderr, " %.17g", hs[J.soff + k]);
      std::fprintf(stderr, "\n");
    }
  // per sector: descending order, relative cut-off 1e-10, cap max_dcut (Dense::svd, src/dense_inst.cpp:497-506)
  std::vector<std::vector<int>> order(jobs.size());
  std::vector<std::vector<double>> ssort(jobs.size());
  std::vector<int> dc(nm1, 0);
  std::vector<double> wsort;
  std::vector<int> isort;
  double wtotal = 0.0;
  for (int i = 0; i < nm1; ++i) {
    if (job_of[i] < 0) continue;
    const SvdJob& J = jobs[job_of[i]];
    const int C = std::min(J.m, J.n);
    auto& o = order[job_of[i]];
    o.resize(C);
    std::iota(o.begin(), o.end(), 0);
    std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return hs[J.soff + a] > hs[J.soff + b]; });
    auto& s = ssort[job_of[i]];
    s.resize(C);
    for (int k = 0; k < C; ++k) { s[k] = hs[J.soff + o[k]]; wtotal += s[k] * s[k]; }
    const double smax = (C > 0 && s[0] > 1e-16) ? s[0] : 1.0;
    int kept = 0;
    for (int k = 0; k < C; ++k)
      if (s[k] / smax > 1e-10) ++kept;
    if (kept == 0) kept = 1;
    if (max_dcut > 0 && kept > max_dcut) kept = max_dcut;
    dc[i] = kept;
    for (int k = 0; k < kept; ++k) { wsort.push_back(s[k]); isort.push_back(i); }
  }
  // global descending sort without tie-break (sort2, src/block_tensor_inst.cpp:38-50)
  {
    std::vector<std::pair<double, int>> tmp(wsort.size());
    for (size_t k = 0; k < wsort.size(); ++k) tmp[k] = {wsort[k], isort[k]};
    std::sort(tmp.begin(), tmp.end(), [](auto& a, auto& b) { return a.first > b.first; });
    for (size_t k = 0; k < wsort.size(); ++k) { wsort[k] = tmp[k].first; isort[k] = tmp[k].second; }
  }
  const int ntot = (int)wsort.size();
  const int dcut = ntot > max_dcut ? max_dcut : ntot;
  if (dcut < ntot && dcut > 0 && std::fabs(wsort[dcut - 1] - wsort[dcut]) <= 1e-8 * wsort[dcut - 1]) out.near_tie = true;
  // the per-sector relative cut-off decided by rounding: a value within two
  // decades of 1e-10 s_max (such values are rounding noise of an exactly
  // rank-deficient block) that the global cut would otherwise keep
  {
    int sure = 0;
    bool grey = false;
    for (size_t j = 0; j < ssort.size(); ++j) {
      const auto& sv = ssort[j];
      const double smax = (!sv.empty() && sv[0] > 1e-16) ? sv[0] : 1.0;
      for (double x : sv) {
        if (x / smax >= 1e-8) ++sure;
        else if (x / smax > 1e-12) grey = true;
      }
    }
    if (grey && sure < max_dcut) out.near_tie = true;
  }
  // gap at the cut relative to the norm of psi (sum of all squared singular values)
  if (dcut < ntot && dcut > 0) {
    double w2 = 0.0;
    for (double x : wsort) w2 += x * x;
    out.cut_gap = (wsort[dcut - 1] - wsort[dcut]) / std::sqrt(std::max(w2, 1e-300));
  }
  std::vector<int> dim(nm1, 0);
  for (int k = 0; k < dcut; ++k) dim[isort[k]]++;
  std::vector<int> amom, bdim;
  double kept_w = 0.0;
  // the singular values in the reference's output order (src/block_tensor_inst.cpp:576-600):
  // the kept ones sector by sector from position 0, then from position dcut the
  // discarded ones of every sector, sector by sector
  if (wout) wout->assign(wsort.size(), 0.0);
  int wm = 0, wm1 = dcut;
  for (int i = 0; i < nm1; ++i) {
    if (job_of[i] < 0) continue;
    const std::vector<double>& ws = ssort[job_of[i]];
    if (dim[i] > 0) {
      amom.push_back(bb0.q[i]);
      bdim.push_back(dim[i]);
      for (int k = 0; k < dim[i]; ++k) kept_w += ws[k] * ws[k];
    }
    if (wout) {
      for (int k = 0; k < dim[i]; ++k) (*wout)[wm++] = ws[k];
      for (int k = dim[i]; k < dc[i]; ++k) (*wout)[wm1++] = ws[k];
    }
  }
  out.kept = dcut;
  out.discarded_weight = wtotal > 0 ? std::max(0.0, 1.0 - kept_w / wtotal) : 0.0;
  Bond nb(bb0.dir, amom, bdim);
  Bond nbv = nb;
  if (c.sym == Sym::U1) nbv.invert();
  Struct su(c.sym, 0, {bb20, bb21, nb}), svs(c.sym, 0, {bb22, bb23, nbv});
  // positions of (x, y) pairs inside each fused sector (BlockTensor::fuse ordering)
  auto fuse_pos = [&](const Bond& a, const Bond& b, const Bond& f) {
    Struct fs(c.sym, 0, {a, b, f});
    std::vector<long long> pos(fs.nten(), -1);
    std::vector<int> acc(f.nmom(), 0);
    int q[8], d[8];
    for (long i = 0; i < fs.nten(); ++i) {
      if (!fs.block(i, q, d)) continue;
      const int k = f.index_of(q[2]);
      pos[i] = acc[k];
      acc[k] += d[0] * d[1];
    }
    return std::make_pair(fs, pos);
  };
  auto fu = fuse_pos(bb20, bb21, bb0), fv = fuse_pos(bb22, bb23, bb1);
  // permutation and sorted singular values for the gathers
  std::vector<int> perm;
  std::vector<double> wsorted;
  std::vector<long long> poff(jobs.size(), 0);
  for (size_t j = 0; j < jobs.size(); ++j) {
    poff[j] = (long long)perm.size();
    perm.insert(perm.end(), order[j].begin(), order[j].end());
    wsorted.insert(wsorted.end(), ssort[j].begin(), ssort[j].end());
  }
  DevBuf dperm(sizeof(int) * std::max<size_t>(perm.size(), 1), c.stream),
      dw(sizeof(double) * std::max<size_t>(wsorted.size(), 1), c.stream);
  if (!perm.empty()) {
    SADMRG_CUDA(cudaMemcpyAsync(dperm.get(), perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice, c.stream));
    SADMRG_CUDA(cudaMemcpyAsync(dw.get(), wsorted.data(), sizeof(double) * wsorted.size(), cudaMemcpyHostToDevice, c.stream));
  }
  auto build = [&](const Struct& st, const std::pair<Struct, std::vector<long long>>& fz, const Bond& fb,
                   bool left) -> BTensor<S> {
    int q[8], d[8];
    std::vector<char> pres(st.nten(), 0);
    std::vector<Gather> gs;
    for (long m = 0; m < st.nten(); ++m) {
      if (!st.block(m, q, d)) continue;
      const int i = bb0.index_of(q[2]);
      if (i < 0 || dim[i] == 0) continue;
      int fq[3] = {q[0], q[1], q[2]};
      if (!fz.first.allowed_labels(fq)) continue;
      const long fi = fz.first.index(fq);
      if (fi < 0 || fz.second[fi] < 0) continue;
      (void)fb;
      pres[m] = 1;
    }
    BTensor<S> t = alloc_tensor<S>(c, st, pres);
    for (long m = 0; m < st.nten(); ++m) {
      if (!pres[m]) continue;
      st.block(m, q, d);
      const int i = bb0.index_of(q[2]);
      const int jb = job_of[i];
      const SvdJob& J = jobs[jb];
      int fq[3] = {q[0], q[1], q[2]};
      const long long pos = fz.second[fz.first.index(fq)];
      Gather g{};
      g.doff = t.off[m];
      g.rows = d[0] * d[1];
      g.kept = dim[i];
      g.woff = poff[jb];
      g.poff = poff[jb];
      if (left) {  // U columns scaled by s^p1
        g.conj = 0;
        if (!J.trans) { g.soff = J.woff + pos; g.lds = J.m; g.p = p1 - 1.0; }
        else          { g.soff = J.voff + pos; g.lds = J.m; g.p = p1; }
      } else {     // conj(V) columns scaled by s^p2
        g.conj = 1;
        if (!J.trans) { g.soff = J.voff + pos; g.lds = J.n; g.p = p2; }
        else          { g.soff = J.woff + pos; g.lds = J.n; g.p = p2 - 1.0; }
      }
      gs.push_back(g);
    }
    if (!gs.empty()) {
      DevBuf dg(sizeof(Gather) * gs.size(), c.stream);
      SADMRG_CUDA(cudaMemcpyAsync(dg.get(), gs.data(), sizeof(Gather) * gs.size(), cudaMemcpyHostToDevice, c.stream));
      launch_gather(kCx<S>, t.data(), wv.get(), dw.as<double>(), dperm.as<int>(), dg.as<Gather>(), (int)gs.size(),
                    c.stream);
      ++c.launches;
      SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    }
    return t;
  };
  BTensor<S> nu = build(su, fu, bb0, true);
  BTensor<S> nv = build(svs, fv, bb1, false);
  tu = std::move(nu);
  tv = std::move(nv);
  return out;
}

// ---------------------------------------------------------------------------
// chain
template <class S>
Chain<S>::Chain(Ctx& cc, int lx_, int ly_, int bondd_, int physpn_, int totspin_, int open, double J2)
    : c(cc), lx(lx_), ly(ly_), ns(lx_ * ly_), bondd(bondd_), physpn(physpn_), totspin(totspin_), max_dcut(bondd_) {
  SADMRG_REQUIRE(ns >= 6 && ns % 2 == 0, SADMRG_ERR_ARG, "chain: need an even number of sites >= 6");
  SADMRG_REQUIRE(physpn == 1, SADMRG_ERR_ARG, "chain: spin-1/2 sites only");
  uu.resize(ns);
  hh.resize(ns);
  opr.assign(ns, std::vector<BTensor<S>>(ns));
  hmap.assign(ns, std::vector<int>(ns, 0));
  fll.assign(ns, std::vector<int>(ns, 0));
  frr.assign(ns, std::vector<int>(ns, 0));
  coup.assign(ns + 1, 0.0);
  // snake-ordered lattice bonds (src/dmrg_inst.cpp:121-144); open = no wrap-around
  auto site = [&](int x, int y) { return (x % 2 == 0) ? x * ly + y : x * ly + (ly - 1 - y); };
  for (int i = 0; i < ns; ++i) {
    const int x1 = i / ly, y1 = (x1 % 2 == 0) ? i % ly : ly - 1 - (i % ly);
    for (int k = 0; k < 2; ++k) {
      int x2 = x1, y2 = y1;
      if (k == 0) { x2 = x1 + 1; if (x2 >= lx) { if (open) continue; x2 %= lx; } }
      else        { y2 = y1 + 1; if (y2 >= ly) { if (open) continue; y2 %= ly; } }
      const int j = site(x2, y2);
      if (i != j) { hmap[i][j] = 1; hmap[j][i] = 1; }
    }
  }
  coup[1] = 1.0;
  if (J2 != 0.0) {
    for (int i = 0; i + 2 < ns; ++i) { hmap[i][i + 2] = 2; hmap[i + 2][i] = 2; }
    coup[2] = J2;
  }
  for (int i = 0; i < ns; ++i) {
    for (int j = 0; j < i; ++j)
      for (int k = i + 1; k < ns; ++k)
        if (hmap[j][k] != 0) fll[i][j] = 1;
    for (int j = i + 1; j < ns; ++j)
      for (int k = 0; k < i; ++k)
        if (hmap[j][k] != 0) frr[i][j] = 1;
  }
  if (c.sym == Sym::SU2 && !c.cgc) c.cgc = std::make_unique<CGCFactors>(physpn);
  init_local_operators();
}

// DMRG::initialize_local_operators (src/dmrg_inst.cpp:222-260) with
// BlockTensor::make_spinor_start (src/block_tensor_inst.cpp:1145-1217)
template <class S>
void Chain<S>::init_local_operators() {
  const int p = physpn;
  if (c.sym == Sym::SU2) {
    Struct st(Sym::SU2, 0, {Bond(-1, {p}, {1}), Bond(-1, {2}, {1}), Bond(1, {p}, {1})});
    const double r = std::sqrt(3.0) / 2.0;
    for (int k = 0; k < 2; ++k) {
      S val = S(k == 0 ? r : -r);
      sigma[k] = ops::from_host<S>(c, st, {1}, &val);
      sigma[k].host = {val};
    }
    return;
  }
  std::vector<int> qs, ones;
  for (int i = 0; i <= p; ++i) { qs.push_back(-p + 2 * i); ones.push_back(1); }
  Bond bp(-1, qs, ones), bk(1, qs, ones);
  Struct s0(Sym::U1, 0, {bp, Bond(-1, {-2, 0, 2}, {1, 1, 1}), bk});
  Struct s1(Sym::U1, 0, {bp, Bond(1, {-2, 0, 2}, {1, 1, 1}), bk});
  for (int k = 0; k < 2; ++k) {
    const Struct& st = k == 0 ? s0 : s1;
    std::vector<char> pres(st.nten(), 0);
    std::vector<S> vals;
    int q[8], d[8];
    for (long i = 0; i < st.nten(); ++i) {
      if (!st.block(i, q, d)) continue;
      // sigma[1] carries the channel charge reversed (contract with fuse_to_singlet + shift)
      const int qc = (k == 0) ? q[1] : -q[1];
      double v;
      if (q[0] == q[2] && qc == 0) v = q[0] / 2.0;
      else if (q[0] != q[2]) v = 1.0 / std::sqrt(2.0);
      else continue;
      pres[i] = 1;
      vals.push_back(S(v));
    }
    sigma[k] = ops::from_host<S>(c, st, pres, vals.data());
    sigma[k].host = vals;
  }
}

// op += (coupling of the pair a < b) * src.  On J1 bonds with a DM term,
// J S_a.S_b + Dz (S_a x S_b)_z = J Sz Sz + (J + i Dz)/2 S+_a S-_b + (J - i Dz)/2 S-_a S+_b,
// and the U(1) channel leg labels these parts: charge -2 pairs S+_a with S-_b
// (sigma[0] holds S+/sqrt2 at channel -2), 0 pairs Sz with Sz, +2 pairs S-_a
// with S+_b; both operators of a pair carry the same label, so weighting the
// summed side's channels by (J + i Dz, J, J - i Dz) adds the term.  Not in the
// reference, whose couplings are one real scalar per pair.
template <class S>
void Chain<S>::add_coupled(BTensor<S>& op, const BTensor<S>& src, int a, int b) {
  const int h = hmap[a][b];
  const double J = coup[h];
  if constexpr (kCx<S>) {
    if (h == 1 && dz != 0.0) {
      const S w[3] = {S(J, dz), S(J, 0.0), S(J, -dz)};
      ops::add_into_channels<S>(c, op, src, w);
      return;
    }
  }
  ops::add_into<S>(c, op, src, S(J));
}

template <class S>
void Chain<S>::set_dm(double d) {
  SADMRG_REQUIRE(d == 0.0 || (c.sym == Sym::U1 && kCx<S>), SADMRG_ERR_ARG,
                 "chain: the DM term needs U(1) symmetry and complex scalars");
  for (int i = 0; i < ns; ++i)
    SADMRG_REQUIRE(uu[i].null() && hh[i].null(), SADMRG_ERR_STATE,
                   "chain: set the DM term before iDMRG or loading a checkpoint");
  dz = d;
}

template <class S>
void Chain<S>::set_excited(int k) {
  SADMRG_REQUIRE(k >= 0 && k <= 16, SADMRG_ERR_ARG, "chain: excited state index 0..16");
  for (int i = 0; i < ns; ++i)
    SADMRG_REQUIRE(uu[i].null() && hh[i].null(), SADMRG_ERR_STATE,
                   "chain: set the excited state before iDMRG or loading a checkpoint");
  exci = k;
  orth.assign(k, std::vector<BTensor<S>>(ns));
  ovlp.assign(k, std::vector<BTensor<S>>(ns));
  low_enr.assign(k, 0.0);
  overlapvec.assign(k, BTensor<S>());
}

template <class S>
void Chain<S>::random_init(BTensor<S>& t) {
  std::vector<S> h(t.nelem);
  for (long long i = 0; i < t.nelem; ++i) {
    if constexpr (kCx<S>) h[i] = S(dist(rng), dist(rng));
    else h[i] = dist(rng);
  }
  if (t.nelem > 0)
    SADMRG_CUDA(cudaMemcpyAsync(t.data(), h.data(), sizeof(S) * t.nelem, cudaMemcpyHostToDevice, c.stream));
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));
}

// DMRG::prepare_site_operator_from_left (src/dmrg_inst.cpp:440-511 and 587-639)
template <class S>
void Chain<S>::prepare_site_operator_from_left(int i, bool real_env, int flag) {
  const double t0 = now_s();
  BTensor<S> u1;
  if (!real_env) u1 = ops::fuse<S>(c, uu[i].st.bonds[0], uu[i].st.bonds[1]);
  const BTensor<S>& U = real_env ? uu[i] : u1;
  if (real_env && i == 0) {
    opr[0][0] = ops::operator_initial<S>(c, U, U, sigma[0], 0);
    for (int j = 0; j < exci; ++j) ovlp[j][0] = ops::overlap_initial<S>(c, orth[j][0], uu[0], 0);
    hh[0] = BTensor<S>();
    timers.env += now_s() - t0;
    return;
  }
  // the lower states' overlap environments (src/dmrg_inst.cpp:495-501); with flag,
  // the lower state's sites i+1 and i+2 in the current bases: the left
  // environment contracted into orth[i+1], orth[i+2] into the right one.  The
  // latter contracts orth's middle leg: BlockTensor::contract lists the remaining
  // bonds cyclically after the contracted one (src/block_tensor_inst.cpp:1067-1071),
  // (orth.2, orth.0, env.1), which the contraction here gives after rotating orth
  // to (orth.2, orth.0, orth.1); BlockTensor::shift(1, 0) then rotates the result
  // to (orth.0, env.1, orth.2), the leg order of the right-side site tensors.
  if (real_env)
    for (int j = 0; j < exci; ++j) {
      ovlp[j][i] = ops::overlap_transformation<S>(c, orth[j][i], uu[i], ovlp[j][i - 1], 0);
      if (flag == 1) {
        ovlp[j][i + 1] = ops::contract<S>(c, ovlp[j][i], 0, orth[j][i + 1], 0);
        static const int cyc[3] = {2, 0, 1}, rot[3] = {1, 2, 0};
        BTensor<S> t = ops::permute3<S>(c, orth[j][i + 2], cyc);
        ovlp[j][i + 2] = ops::permute3<S>(c, ops::contract<S>(c, t, 2, ovlp[j][i + 3], 0), rot);
      }
    }
  BTensor<S> hnew;
  if (!hh[i - 1].null()) hnew = ops::overlap_transformation<S>(c, U, U, hh[i - 1], 0);
  std::vector<BTensor<S>> newopr(i);
  for (int k = 0; k < i; ++k)
    if (fll[i][k] == 1) newopr[k] = ops::operator_transformation<S>(c, U, U, opr[i - 1][k], 0);
  BTensor<S> op;
  for (int m = 0; m < i; ++m)
    if (hmap[i][m] > 0) add_coupled(op, opr[i - 1][m], m, i);
  if (!op.null()) {
    BTensor<S> ht = ops::operator_pairup<S>(c, U, U, op, sigma[1], 0);
    ops::add_into<S>(c, hnew, ht, S(1.0));
  }
  for (int k = 0; k < i; ++k)
    if (fll[i][k] == 1) opr[i][k] = std::move(newopr[k]);
  opr[i][i] = ops::operator_initial<S>(c, U, U, sigma[0], 0);
  hh[i] = std::move(hnew);
  timers.env += now_s() - t0;
}

// DMRG::prepare_site_operator_from_right (src/dmrg_inst.cpp:515-583 and 643-695)
template <class S>
void Chain<S>::prepare_site_operator_from_right(int i, bool real_env, int flag) {
  const double t0 = now_s();
  BTensor<S> u1;
  if (!real_env) u1 = ops::fuse<S>(c, uu[i].st.bonds[0], uu[i].st.bonds[1]);
  const BTensor<S>& U = real_env ? uu[i] : u1;
  if (real_env && i == ns - 1) {
    opr[i][i] = ops::operator_initial<S>(c, U, U, sigma[1], 1);
    for (int j = 0; j < exci; ++j) ovlp[j][i] = ops::overlap_initial<S>(c, orth[j][i], uu[i], 1);
    hh[i] = BTensor<S>();
    timers.env += now_s() - t0;
    return;
  }
  // the mirror image of the left update (src/dmrg_inst.cpp:567-573)
  if (real_env)
    for (int j = 0; j < exci; ++j) {
      ovlp[j][i] = ops::overlap_transformation<S>(c, orth[j][i], uu[i], ovlp[j][i + 1], 1);
      if (flag == 1) {
        ovlp[j][i - 2] = ops::contract<S>(c, ovlp[j][i - 3], 0, orth[j][i - 2], 0);
        static const int cyc[3] = {2, 0, 1}, rot[3] = {1, 2, 0};
        BTensor<S> t = ops::permute3<S>(c, orth[j][i - 1], cyc);
        ovlp[j][i - 1] = ops::permute3<S>(c, ops::contract<S>(c, t, 2, ovlp[j][i], 0), rot);
      }
    }
  BTensor<S> hnew;
  if (!hh[i + 1].null()) hnew = ops::overlap_transformation<S>(c, U, U, hh[i + 1], 1);
  std::vector<BTensor<S>> newopr(ns);
  for (int m = 0; m < ns - 1 - i; ++m) {
    const int k = i + 1 + m;
    if (frr[i][k] == 1) newopr[k] = ops::operator_transformation<S>(c, U, U, opr[i + 1][k], 1);
  }
  BTensor<S> op;
  for (int m = 0; m < ns - 1 - i; ++m) {
    const int k = i + 1 + m;
    if (hmap[i][k] > 0) add_coupled(op, opr[i + 1][k], i, k);
  }
  if (!op.null()) {
    BTensor<S> ht = ops::operator_pairup<S>(c, U, U, op, sigma[0], 1);
    ops::add_into<S>(c, hnew, ht, S(1.0));
  }
  for (int m = 0; m < ns - 1 - i; ++m) {
    const int k = i + 1 + m;
    if (frr[i][k] == 1) opr[i][k] = std::move(newopr[k]);
  }
  opr[i][i] = ops::operator_initial<S>(c, U, U, sigma[1], 1);
  hh[i] = std::move(hnew);
  timers.env += now_s() - t0;
}

// DMRG::prepare_input_vector (src/dmrg_inst.cpp:412-437)
template <class S>
void Chain<S>::prepare_input_vector(int il, int ir, BTensor<S>& vec) {
  const double t0 = now_s();
  BTensor<S> t1 = ops::fuse<S>(c, uu[il].st.bonds[0], uu[il].st.bonds[1]);
  BTensor<S> t2 = ops::fuse<S>(c, uu[ir].st.bonds[0], uu[ir].st.bonds[1]);
  BTensor<S> left = ops::overlap_initial<S>(c, uu[il], t1, 0);
  BTensor<S> rght = ops::overlap_initial<S>(c, uu[ir], t2, 1);
  if (c.sym == Sym::SU2) ops::take_conjugate(left, 0);
  vec = ops::contract<S>(c, left, 0, rght, 0);
  ops::makeup_input_vector<S>(c, vec);
  // the lower states in the same two-site basis (src/dmrg_inst.cpp:429-436)
  if (il + 1 == ir)
    for (int j = 0; j < exci; ++j) {
      BTensor<S> lj = ops::overlap_initial<S>(c, ovlp[j][il], t1, 0);
      BTensor<S> rj = ops::overlap_initial<S>(c, ovlp[j][ir], t2, 1);
      if (c.sym == Sym::SU2) ops::take_conjugate(lj, 0);
      overlapvec[j] = ops::contract<S>(c, lj, 0, rj, 0);
      ops::makeup_input_vector<S>(c, overlapvec[j]);
    }
  timers.prep += now_s() - t0;
}

// DMRG::prepare_input_vector_initial (src/dmrg_inst.cpp:375-410)
template <class S>
void Chain<S>::prepare_input_vector_initial(int il, int ir, BTensor<S>& vec) {
  const double t0 = now_s();
  BTensor<S> t1 = ops::fuse<S>(c, uu[il].st.bonds[0], uu[il].st.bonds[1]);
  BTensor<S> t2 = ops::fuse<S>(c, uu[ir].st.bonds[0], uu[ir].st.bonds[1]);
  BTensor<S> left = ops::overlap_initial<S>(c, uu[il], t1, 0);
  BTensor<S> rght = ops::overlap_initial<S>(c, uu[ir], t2, 1);
  Bond b0 = left.st.bonds[0], b1 = rght.st.bonds[0];
  b0.invert();
  b1.invert();
  BTensor<S> tmp = ops::fuse_to_singlet<S>(c, b0, b1);
  BTensor<S> tmp3 = ops::contract<S>(c, left, 0, tmp, 0);
  vec = ops::contract<S>(c, tmp3, 1, rght, 0);
  ops::makeup_input_vector<S>(c, vec);
  timers.prep += now_s() - t0;
}

// operator set of DMRG::hamiltonian_vector_multiplication_idmrg (src/dmrg_inst.cpp:309-351)
template <class S>
HeffPlan<S> Chain<S>::heff_plan(int il, int ir, const BTensor<S>& vec, bool tune) {
  std::vector<const BTensor<S>*> opl;
  std::vector<BTensor<S>> sums;
  sums.reserve(ns);
  std::vector<PairTerm> terms;
  int m1, m4;
  if (il < ns / 2) { m1 = il + 1; m4 = ns - ir; }
  else { m1 = ns - ir; m4 = il + 1; }
  for (int m0 = 0; m0 < m1; ++m0) {
    int j = 0, k = 0;
    if (il < ns / 2) j = m0;
    else k = ir + m0;
    BTensor<S> op;
    for (int m = 0; m < m4; ++m) {
      if (il < ns / 2) k = ir + m;
      else j = m;
      if (hmap[j][k] > 0) add_coupled(op, il < ns / 2 ? opr[ir][k] : opr[il][j], j, k);
    }
    if (op.null()) continue;
    sums.push_back(std::move(op));
    const BTensor<S>* fixed = (il < ns / 2) ? &opr[il][j] : &opr[ir][k];
    if (fixed->null()) continue;
    PairTerm t;
    opl.push_back(fixed);
    const int fi = (int)opl.size() - 1;
    opl.push_back(&sums.back());
    const int si = (int)opl.size() - 1;
    if (il < ns / 2) { t.op1 = fi; t.op2 = si; }
    else { t.op1 = si; t.op2 = fi; }
    terms.push_back(t);
  }
  return build_heff<S>(c, vec, hh[il].null() ? nullptr : &hh[il], hh[ir].null() ? nullptr : &hh[ir], opl, terms,
                       tune);
}

// DMRG::lanczos_solve_eigenvector_idmrg (src/dmrg_inst.cpp:264-279)
// The excited-state penalty of DMRG::hamiltonian_vector_multiplication_idmrg
// (src/dmrg_inst.cpp:352-363): out -= sum_j gs_enr[j] <overlapvec[j]|psi> overlapvec[j]
// over the lower states j, their projections taken into psi's block layout (both
// are built on the same fused bonds, so a block present in one is at the same
// index in the other).
template <class S>
void Chain<S>::set_penalty(HeffPlan<S>& H, const BTensor<S>& vec) {
  const size_t bytes = sizeof(S) * (size_t)H.n * exci;
  H.pen_o = std::make_shared<DevBuf>(bytes, c.stream);
  H.pen_wo = std::make_shared<DevBuf>(bytes, c.stream);
  H.pen_dot = std::make_shared<DevBuf>(sizeof(S) * (exci + 1), c.stream);
  SADMRG_CUDA(cudaMemsetAsync(H.pen_o->get(), 0, bytes, c.stream));
  int q[8], d[8], qo[8], dn[8];
  for (int j = 0; j < exci; ++j) {
    const BTensor<S>& o = overlapvec[j];
    SADMRG_REQUIRE(!o.null() && o.nten() == vec.nten() && o.st.nbond() == vec.st.nbond(), SADMRG_ERR_STATE,
                   "excited state: the lower state's projection does not match the two-site basis");
    S* dst = static_cast<S*>(H.pen_o->get()) + (size_t)j * H.n;
    for (long b = 0; b < vec.nten(); ++b) {
      if (!vec.present(b) || !o.present(b) || !vec.st.block(b, q, d)) continue;
      o.st.block(b, qo, dn);
      for (int k = 0; k < vec.st.nbond(); ++k)
        SADMRG_REQUIRE(qo[k] == q[k] && dn[k] == d[k], SADMRG_ERR_STATE,
                       "excited state: a block of the lower state's projection has other sectors or dims");
      SADMRG_CUDA(cudaMemcpyAsync(dst + vec.off[b], o.data() + o.off[b], sizeof(S) * vec.st.block_elems(b),
                                  cudaMemcpyDeviceToDevice, c.stream));
    }
  }
  SADMRG_CUDA(cudaMemcpyAsync(H.pen_wo->get(), H.pen_o->get(), bytes, cudaMemcpyDeviceToDevice, c.stream));
  for (int j = 0; j < exci; ++j)
    launch_scale(kCx<S>, static_cast<S*>(H.pen_wo->get()) + (size_t)j * H.n, low_enr[j], 0.0, H.n, c.stream);
  H.npen = exci;
}

template <class S>
void Chain<S>::lanczos_solve_eigenvector(int il, int ir, BTensor<S>& vec) {
  const double t0 = now_s();
  int mlanc = mlanc_max;
  long long ndata = 0;
  {
    int q[8], d[8];
    for (long i = 0; i < vec.nten(); ++i)
      if (vec.st.block(i, q, d)) ndata += vec.st.block_elems(i);
  }
  if (mlanc > ndata) mlanc = (int)ndata + 1;
  if (mlanc < 2) mlanc = 2;
  const double tp = now_s();
  HeffPlan<S> H = heff_plan(il, ir, vec);
  timers.plan += now_s() - tp;
  if (exci > 0 && il + 1 == ir) set_penalty(H, vec);
  LanczosStats st = lanczos_solve<S>(c, H, vec.data(), mlanc, prec);
  gs_enr = st.energy;
  if (std::getenv("SADMRG_VERBOSE"))
    std::fprintf(stderr, "lanczos (%d,%d) E=%.15f matvecs=%d ov=%.3e n=%lld\n", il, ir, st.energy, st.matvecs,
                 st.overlap, (long long)vec.nelem);
  timers.matvecs += st.matvecs;
  timers.heff_flops += (double)H.flops * st.matvecs;
  timers.lanczos += now_s() - t0;
}

template <class S>
void Chain<S>::wavefunc_transformation(int i, int dir) {
  const double t0 = now_s();
  if (dir == 0) ops::right2left_vectran<S>(c, uu[i]);
  else ops::left2right_vectran<S>(c, uu[i]);
  for (int j = 0; j < exci; ++j) {   // src/dmrg_inst.cpp:862-868
    if (dir == 0) ops::right2left_vectran<S>(c, orth[j][i]);
    else ops::left2right_vectran<S>(c, orth[j][i]);
  }
  timers.prep += now_s() - t0;
}

template <class S>
void Chain<S>::svd_step(BTensor<S>& vec, int il, int ir, double p1, double p2) {
  const double t0 = now_s();
  std::vector<double> w;
  SvdStats s = block_svd<S>(c, vec, uu[il], p1, uu[ir], p2, max_dcut, &w);
  // BlockTensor::svd overwrites the first n values of the chain's ww array and
  // leaves the rest as it was (src/block_tensor_inst.cpp:576-600)
  if (ww.size() < w.size()) ww.resize(w.size(), 0.0);
  std::copy(w.begin(), w.end(), ww.begin());
  last_discarded = s.discarded_weight;
  if (s.near_tie) ++near_ties;
  {
    int f = s.near_tie ? 1 : 0;
    if (s.cut_gap < 10.0 * std::sqrt(c.lanczos_ov_tol)) f |= 2;
    if ((int)bond_flags.size() < ns) bond_flags.assign(ns, 0);
    bond_flags[il] = f;
  }
  // the stop test fixes the Ritz vector only to about sqrt(ov_tol) (times |E| / gap),
  // so a cut whose gap is within that of 0 can fall either way in two correct runs
  if (s.cut_gap < 10.0 * std::sqrt(c.lanczos_ov_tol)) ++stop_ties;
  if (s.jacobi_kernel_ms > 0) timers.svd_kernel += s.jacobi_kernel_ms * 1e-3;
  timers.svd_sweeps += s.sweeps_max > 0 ? s.sweeps_max : 0;
  if (std::getenv("SADMRG_VERBOSE")) {
    std::fprintf(stderr, "svd (%d,%d) kept=%d dw=%.3e sweeps=%d jacobi=%.2fms kernel=%.2fms max=%dx%d total=%.2fms sectors:",
                 il, ir, s.kept, s.discarded_weight, s.sweeps_max, s.jacobi_s * 1e3, s.jacobi_kernel_ms, s.max_rows,
                 s.max_cols,
                 (now_s() - t0) * 1e3);
    const Bond& b = uu[il].st.bonds[2];
    for (int k = 0; k < b.nmom(); ++k) std::fprintf(stderr, " %d:%d", b.q[k], b.d[k]);
    std::fprintf(stderr, "\n");
  }
  timers.svd += now_s() - t0;
}

// boundary tensors (src/dmrg_inst.cpp:710-740 and 812-840)
template <class S>
static void edge_tensors(Chain<S>& ch, Bond& bphys_l, Bond& bphys_r) {
  Ctx& c = ch.c;
  Bond b0, b3;
  if (c.sym == Sym::SU2) {
    b0 = Bond(1, {0}, {1});
    bphys_l = Bond(1, {ch.physpn}, {1});
    bphys_r = Bond(1, {ch.physpn}, {1});
    b3 = Bond(1, {ch.totspin}, {1});
  } else {
    b0 = Bond(1, {0}, {1});
    bphys_l = Bond(1, {-1, 1}, {1, 1});
    bphys_r = Bond(1, {-1, 1}, {1, 1});
    b3 = Bond(-1, {ch.totspin}, {1});
  }
  ch.uu[0] = ops::fuse<S>(c, b0, bphys_l);
  ch.uu[ch.ns - 1] = ops::fuse<S>(c, bphys_r, b3);
}

// DMRG::do_idmrg (src/dmrg_inst.cpp:699-804)
template <class S>
void Chain<S>::do_idmrg() {
  SADMRG_REQUIRE(exci == 0, SADMRG_ERR_STATE, "chain: an excited state starts from read_mps, not iDMRG");
  Bond bl, br;
  edge_tensors(*this, bl, br);
  BTensor<S> vec;
  for (int i = 0; i <= ns / 2 - 2; ++i) {
    prepare_site_operator_from_left(i, true);
    prepare_site_operator_from_right(ns - 1 - i, true);
    Bond b0 = uu[i].st.bonds[2], b1 = uu[ns - 1 - i].st.bonds[2];
    b0.invert();
    b1.invert();
    uu[i + 1] = ops::fuse<S>(c, b0, bl);
    uu[ns - 2 - i] = ops::fuse<S>(c, br, b1);
    if (((i + 2) * 2 * physpn >= totspin && i >= 1) || i == ns / 2 - 2) {
      prepare_input_vector_initial(i + 1, ns - 2 - i, vec);
      prepare_site_operator_from_left(i + 1, false);
      prepare_site_operator_from_right(ns - 2 - i, false);
      random_init(vec);
      lanczos_solve_eigenvector(i + 1, ns - 2 - i, vec);
      if (i == ns / 2 - 2) svd_step(vec, i + 1, ns - 2 - i, 1.0, 0.0);
      else svd_step(vec, i + 1, ns - 2 - i, 0.0, 0.0);
    }
  }
}

// DMRG::prepare_sweep (src/dmrg_inst.cpp:808-854)
template <class S>
void Chain<S>::prepare_sweep() {
  Bond bl, br;
  edge_tensors(*this, bl, br);
  for (int i = 0; i < ns / 2 - 1; ++i) {
    prepare_site_operator_from_left(i, true, 0);
    prepare_site_operator_from_right(ns - 1 - i, true, i < ns / 2 - 2 ? 0 : 1);
  }
}

// DMRG::sweep (src/dmrg_inst.cpp:874-943)
template <class S>
void Chain<S>::sweep() {
  BTensor<S> vec;
  for (int i = ns / 2; i >= nfree + 2; --i) {
    wavefunc_transformation(i - 1, 1);
    prepare_site_operator_from_right(i, true, 1);
    prepare_input_vector(i - 2, i - 1, vec);
    prepare_site_operator_from_left(i - 2, false);
    prepare_site_operator_from_right(i - 1, false);
    lanczos_solve_eigenvector(i - 2, i - 1, vec);
    if (i > nfree + 2) svd_step(vec, i - 2, i - 1, 1.0, 0.0);
    else svd_step(vec, i - 2, i - 1, 0.0, 1.0);
  }
  for (int i = nfree; i < ns - nfree - 2; ++i) {
    wavefunc_transformation(i + 1, 0);
    prepare_site_operator_from_left(i, true, 1);
    prepare_input_vector(i + 1, i + 2, vec);
    prepare_site_operator_from_left(i + 1, false);
    prepare_site_operator_from_right(i + 2, false);
    lanczos_solve_eigenvector(i + 1, i + 2, vec);
    if (i < ns - nfree - 3) svd_step(vec, i + 1, i + 2, 0.0, 1.0);
    else svd_step(vec, i + 1, i + 2, 1.0, 0.0);
  }
  for (int i = ns - nfree - 1; i >= ns / 2 + 1; --i) {
    wavefunc_transformation(i - 1, 1);
    prepare_site_operator_from_right(i, true, 1);
    prepare_input_vector(i - 2, i - 1, vec);
    prepare_site_operator_from_left(i - 2, false);
    prepare_site_operator_from_right(i - 1, false);
    lanczos_solve_eigenvector(i - 2, i - 1, vec);
    std::fill(ww.begin(), ww.begin() + std::min<size_t>(ww.size(), bondd), 0.0);   // src/dmrg_inst.cpp:934
    svd_step(vec, i - 2, i - 1, 1.0, 0.0);
  }
}

// DMRG::read_mps (src/dmrg_inst.cpp:1031-1079): this state's site tensors,
// uu-<ns>-<D>-<2S>-<exci>-<i>; for an excited state also, as
// DMRG::read_mps(read1, read2) (:1081-1140), the lower states idx < exci into orth
// and their last energies from enr-<ns>-<D>-<2S>-<idx>.dat
template <class S>
bool Chain<S>::read_mps(const std::string& dir, int bond_read) {
  if (!read_state(dir, bond_read, exci, uu)) return false;
  for (int idx = 0; idx < exci; ++idx) {
    SADMRG_REQUIRE(read_state(dir, bond_read, idx, orth[idx]), SADMRG_ERR_ARG,
                   "read_mps: lower state " + std::to_string(idx) + " not found in " + dir);
    const std::string name = dir + "/enr-" + std::to_string(ns) + "-" + std::to_string(bond_read) + "-" +
                             std::to_string(totspin) + "-" + std::to_string(idx) + ".dat";
    FILE* f = std::fopen(name.c_str(), "r");
    SADMRG_REQUIRE(f, SADMRG_ERR_ARG, "read_mps: no energy of lower state " + std::to_string(idx) + " (" + name + ")");
    double e;
    bool any = false;
    while (std::fscanf(f, "%lf", &e) == 1) { low_enr[idx] = e; any = true; }
    std::fclose(f);
    SADMRG_REQUIRE(any, SADMRG_ERR_ARG, "read_mps: empty " + name);
  }
  return true;
}

template <class S>
bool Chain<S>::read_state(const std::string& dir, int bond_read, int idx, std::vector<BTensor<S>>& out) {
  out.resize(ns);
  for (int i = 0; i < ns; ++i) {
    const std::string base = dir + "/uu-" + std::to_string(ns) + "-" + std::to_string(bond_read) + "-" +
                             std::to_string(totspin) + "-" + std::to_string(idx) + "-" + std::to_string(i);
    FILE* f = std::fopen((base + ".dat").c_str(), "r");
    if (!f) return false;
    int nb = 0, lc = 0;
    std::vector<Bond> bonds;
    bool ok = std::fscanf(f, "%d %d", &nb, &lc) == 2 && nb >= 1 && nb <= 4;
    for (int b = 0; ok && b < nb; ++b) {
      int dir_ = 0, nc = 0;
      ok = std::fscanf(f, "%d %d", &dir_, &nc) == 2 && nc >= 1 && nc <= (1 << 16);
      std::vector<int> q(ok ? nc : 0), d(ok ? nc : 0);
      for (int k = 0; ok && k < nc; ++k) ok = std::fscanf(f, "%d", &q[k]) == 1;
      for (int k = 0; ok && k < nc; ++k) ok = std::fscanf(f, "%d", &d[k]) == 1 && d[k] >= 1 && d[k] <= (1 << 20);
      if (ok) bonds.push_back(Bond(dir_, q, d));
    }
    std::fclose(f);
    SADMRG_REQUIRE(ok, SADMRG_ERR_ARG, "read_mps: malformed " + base + ".dat");
    Struct st(c.sym, lc, bonds);
    std::vector<char> pres(st.nten(), 0);
    long long ndata = 0;
    int q[8], d[8];
    for (long b = 0; b < st.nten(); ++b)
      if (st.block(b, q, d)) { pres[b] = 1; ndata += st.block_elems(b); }
    std::vector<S> data(ndata);
    FILE* fb = std::fopen((base + ".bin").c_str(), "rb");
    if (!fb) return false;
    const size_t got = std::fread(data.data(), sizeof(S), ndata, fb);
    std::fclose(fb);
    SADMRG_REQUIRE((long long)got == ndata, SADMRG_ERR_ARG, "read_mps: short " + base + ".bin");
    out[i] = ops::from_host<S>(c, st, pres, data.data());
  }
  return true;
}

template <class S>
void Chain<S>::save_mps(const std::string& dir) const {
  for (int i = 0; i < ns; ++i) {
    const BTensor<S>& t = uu[i];
    const std::string base = dir + "/uu-" + std::to_string(ns) + "-" + std::to_string(bondd) + "-" +
                             std::to_string(totspin) + "-" + std::to_string(exci) + "-" + std::to_string(i);
    FILE* f = std::fopen((base + ".dat").c_str(), "w");
    SADMRG_REQUIRE(f, SADMRG_ERR_ARG, "save_mps: cannot write " + base + ".dat");
    std::fprintf(f, "%d\t%d\n", t.st.nbond(), t.st.locspin);
    for (auto& b : t.st.bonds) {
      std::fprintf(f, "%d\t%d\n", b.dir, b.nmom());
      for (int k = 0; k < b.nmom(); ++k) std::fprintf(f, "%d\t", b.q[k]);
      std::fprintf(f, "\n");
      for (int k = 0; k < b.nmom(); ++k) std::fprintf(f, "%d\t", b.d[k]);
      std::fprintf(f, "\n");
    }
    std::fclose(f);
    // data of the allowed blocks (null ones written as zeros), then the SU(2) CGC blocks
    std::vector<S> h = ops::to_host<S>(c, t);
    FILE* fb = std::fopen((base + ".bin").c_str(), "wb");
    SADMRG_REQUIRE(fb, SADMRG_ERR_ARG, "save_mps: cannot write " + base + ".bin");
    int q[8], d[8];
    std::vector<double> cg;
    for (long b = 0; b < t.nten(); ++b) {
      if (!t.st.block(b, q, d)) continue;
      const long long n = t.st.block_elems(b);
      if (t.present(b)) std::fwrite(h.data() + t.off[b], sizeof(S), n, fb);
      else { std::vector<S> z(n, S(0)); std::fwrite(z.data(), sizeof(S), n, fb); }
      if (c.sym == Sym::SU2 && t.st.nbond() == 3) {
        HDense cc;
        cc.make_cgc(q[0], q[1], q[2]);
        cg.insert(cg.end(), cc.v.begin(), cc.v.end());
      }
    }
    if (!cg.empty()) std::fwrite(cg.data(), sizeof(double), cg.size(), fb);
    std::fclose(fb);
  }
}

// DMRG::save_ww (src/dmrg_inst.cpp:1145-1153): bondd * phdim doubles of the ww
// array, ww-<ns>-<bondd>-<2S>-<exci>.bin (the array is kept at least that long here,
// zero beyond what the truncations wrote)
template <class S>
void Chain<S>::save_ww(const std::string& dir) const {
  const std::string name = dir + "/ww-" + std::to_string(ns) + "-" + std::to_string(bondd) + "-" +
                           std::to_string(totspin) + "-" + std::to_string(exci) + ".bin";
  std::vector<double> w((size_t)bondd * (physpn + 1), 0.0);
  std::copy(ww.begin(), ww.begin() + std::min(ww.size(), w.size()), w.begin());
  FILE* f = std::fopen(name.c_str(), "wb");
  SADMRG_REQUIRE(f, SADMRG_ERR_ARG, "save_ww: cannot write " + name);
  const size_t put = std::fwrite(w.data(), sizeof(double), w.size(), f);
  std::fclose(f);
  SADMRG_REQUIRE(put == w.size(), SADMRG_ERR_ARG, "save_ww: short write " + name);
}

// DMRG::read_ww (src/dmrg_inst.cpp:1156-1165): the first read1 doubles of
// ww-<ns>-<read1>-<2S>-<exci>.bin, or read1 ones when the file is absent
template <class S>
void Chain<S>::read_ww(const std::string& dir, int read1) {
  const std::string name = dir + "/ww-" + std::to_string(ns) + "-" + std::to_string(read1) + "-" +
                           std::to_string(totspin) + "-" + std::to_string(exci) + ".bin";
  if (ww.size() < (size_t)read1) ww.resize(read1, 0.0);
  FILE* f = std::fopen(name.c_str(), "rb");
  if (!f) {
    std::fill(ww.begin(), ww.begin() + read1, 1.0);
    return;
  }
  const size_t got = std::fread(ww.data(), sizeof(double), read1, f);
  std::fclose(f);
  SADMRG_REQUIRE(got == (size_t)read1, SADMRG_ERR_ARG, "read_ww: short " + name);
}

// DMRG::save_enr (src/dmrg_inst.cpp:996-1003): appends gs_enr to
// enr-<ns>-<bondd>-<2S>-0.dat, 16 significant digits
template <class S>
void Chain<S>::save_enr(const std::string& dir) const {
  const std::string name = dir + "/enr-" + std::to_string(ns) + "-" + std::to_string(bondd) + "-" +
                           std::to_string(totspin) + "-" + std::to_string(exci) + ".dat";
  FILE* f = std::fopen(name.c_str(), "a");
  SADMRG_REQUIRE(f, SADMRG_ERR_ARG, "save_enr: cannot write " + name);
  std::fprintf(f, "%.16g\n", gs_enr);
  std::fclose(f);
}

// DMRG::read_enr (src/dmrg_inst.cpp:1008-1016): gs_enr = the last value of
// enr-<ns>-<read1>-<2S>-<exci>.dat; unchanged when the file is absent
template <class S>
void Chain<S>::read_enr(const std::string& dir, int read1) {
  const std::string name = dir + "/enr-" + std::to_string(ns) + "-" + std::to_string(read1) + "-" +
                           std::to_string(totspin) + "-" + std::to_string(exci) + ".dat";
  FILE* f = std::fopen(name.c_str(), "r");
  if (!f) return;
  double e;
  while (std::fscanf(f, "%lf", &e) == 1) gs_enr = e;
  std::fclose(f);
}

template <class S>
HeffPlan<S> Chain<S>::freeze(int il, BTensor<S>& psi) {
  SADMRG_REQUIRE(il >= 1 && il + 2 < ns, SADMRG_ERR_ARG, "freeze: bond out of range");
  const int ir = il + 1;
  prepare_input_vector(il, ir, psi);
  prepare_site_operator_from_left(il, false);
  prepare_site_operator_from_right(ir, false);
  return heff_plan(il, ir, psi, /*tune=*/true);
}

template <class S>
static void write_tensor(Ctx& c, const BTensor<S>& t, const std::string& base) {
  FILE* f = std::fopen((base + ".txt").c_str(), "w");
  SADMRG_REQUIRE(f, SADMRG_ERR_ARG, "export: cannot write " + base);
  std::fprintf(f, "nbond %d locspin %d nten %ld\n", t.st.nbond(), t.st.locspin, t.nten());
  for (int b = 0; b < t.st.nbond(); ++b) {
    const Bond& bd = t.st.bonds[b];
    std::fprintf(f, "bond %d dir %d nmom %d q", b, bd.dir, bd.nmom());
    for (int k = 0; k < bd.nmom(); ++k) std::fprintf(f, " %d", bd.q[k]);
    std::fprintf(f, " d");
    for (int k = 0; k < bd.nmom(); ++k) std::fprintf(f, " %d", bd.d[k]);
    std::fprintf(f, "\n");
  }
  int q[8], d[8];
  for (long i = 0; i < t.nten(); ++i) {
    if (!t.present(i)) continue;
    t.st.block(i, q, d);
    std::fprintf(f, "block %ld q", i);
    for (int b = 0; b < t.st.nbond(); ++b) std::fprintf(f, " %d", q[b]);
    std::fprintf(f, " d");
    for (int b = 0; b < t.st.nbond(); ++b) std::fprintf(f, " %d", d[b]);
    std::fprintf(f, " off %lld n %lld\n", (long long)t.off[i], (long long)t.st.block_elems(i));
  }
  std::fclose(f);
  std::vector<S> h = ops::to_host<S>(c, t);
  FILE* fb = std::fopen((base + ".bin").c_str(), "wb");
  SADMRG_REQUIRE(fb, SADMRG_ERR_ARG, "export: cannot write " + base);
  if (!h.empty()) std::fwrite(h.data(), sizeof(S), h.size(), fb);
  std::fclose(fb);
}

template <class S>
void Chain<S>::export_problem(int il, const BTensor<S>& psi, const std::string& dir) const {
  const int ir = il + 1;
  write_tensor(c, psi, dir + "/psi");
  if (!hh[il].null()) write_tensor(c, hh[il], dir + "/hh_il");
  if (!hh[ir].null()) write_tensor(c, hh[ir], dir + "/hh_ir");
  for (int k = 0; k < ns; ++k) {
    if (k <= il && !opr[il][k].null()) write_tensor(c, opr[il][k], dir + "/opr_il_" + std::to_string(k));
    if (k >= ir && !opr[ir][k].null()) write_tensor(c, opr[ir][k], dir + "/opr_ir_" + std::to_string(k));
  }
  FILE* f = std::fopen((dir + "/meta.txt").c_str(), "w");
  SADMRG_REQUIRE(f, SADMRG_ERR_ARG, "export: cannot write meta");
  std::fprintf(f, "sym %d cplx %d ns %d lx %d ly %d D %d sec %d il %d ir %d J2 %.17g open 1 maxangm 0 dz %.17g\n",
               c.sym == Sym::SU2 ? 1 : 0, kCx<S> ? 1 : 0, ns, lx, ly, bondd, totspin, il, ir, coup[2], dz);
  std::fprintf(f, "coup");
  for (int k = 0; k <= ns / 2; ++k) std::fprintf(f, " %.17g", coup[k]);
  std::fprintf(f, "\n");
  for (int a = 0; a < ns; ++a)
    for (int b = 0; b < ns; ++b)
      if (hmap[a][b]) std::fprintf(f, "hmap %d %d %d\n", a, b, hmap[a][b]);
  std::fclose(f);
}

template struct HeffPlan<double>;
template struct HeffPlan<dcmplex>;
template HeffPlan<double> build_heff<double>(Ctx&, const BTensor<double>&, const BTensor<double>*,
                                             const BTensor<double>*, const std::vector<const BTensor<double>*>&,
                                             const std::vector<PairTerm>&, bool);
template HeffPlan<dcmplex> build_heff<dcmplex>(Ctx&, const BTensor<dcmplex>&, const BTensor<dcmplex>*,
                                               const BTensor<dcmplex>*, const std::vector<const BTensor<dcmplex>*>&,
                                               const std::vector<PairTerm>&, bool);
template LanczosStats lanczos1<double>(Ctx&, const HeffPlan<double>&, double*, int, int, bool, int, bool);
template LanczosStats lanczos1<dcmplex>(Ctx&, const HeffPlan<dcmplex>&, dcmplex*, int, int, bool, int, bool);
template LanczosStats lanczos2<double>(Ctx&, const HeffPlan<double>&, double*, int);
template LanczosStats lanczos2<dcmplex>(Ctx&, const HeffPlan<dcmplex>&, dcmplex*, int);
template LanczosStats lanczos_solve<double>(Ctx&, const HeffPlan<double>&, double*, int, int);
template LanczosStats lanczos_solve<dcmplex>(Ctx&, const HeffPlan<dcmplex>&, dcmplex*, int, int);
template SvdStats block_svd<double>(Ctx&, const BTensor<double>&, BTensor<double>&, double, BTensor<double>&, double,
                                    int, std::vector<double>*);
template SvdStats block_svd<dcmplex>(Ctx&, const BTensor<dcmplex>&, BTensor<dcmplex>&, double, BTensor<dcmplex>&,
                                     double, int, std::vector<double>*);
template class Chain<double>;
template class Chain<dcmplex>;

}  // namespace sadmrg
