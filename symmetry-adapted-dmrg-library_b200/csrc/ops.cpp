// ops.cpp -- block-sparse operations of the reference, lowered to device task lists.
#include "ops.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>

namespace sadmrg {

Ctx::~Ctx() {
  if (d_scalars) cudaFree(d_scalars);
  if (d_partial) cudaFree(d_partial);
  if (d_counter) cudaFree(d_counter);
  if (h_pinned) cudaFreeHost(h_pinned);
}

// ---------------------------------------------------------------------------
// tensors
template <class S>
std::vector<Blk> blocks_of(const BTensor<S>& t) {
  std::vector<Blk> v;
  const int nb = t.st.nbond();
  for (long i = 0; i < t.nten(); ++i) {
    if (t.off[i] < 0) continue;
    Blk b{};
    b.idx = i;
    int q[8], d[8];
    t.st.block(i, q, d);
    for (int k = 0; k < 4; ++k) { b.q[k] = k < nb ? q[k] : 0; b.d[k] = k < nb ? d[k] : 1; }
    b.off = t.off[i];
    v.push_back(b);
  }
  return v;
}

template <class S>
BTensor<S> alloc_tensor(Ctx& c, const Struct& st, const std::vector<char>& present) {
  BTensor<S> t;
  t.st = st;
  const long nt = st.nten();
  t.off.assign(nt, -1);
  long long n = 0;
  for (long i = 0; i < nt; ++i)
    if (present[i]) { t.off[i] = n; n += st.block_elems(i); }
  t.nelem = n;
  t.buf = std::make_shared<DevBuf>();
  if (n > 0) {
    t.buf->alloc(sizeof(S) * n, c.stream);
    SADMRG_CUDA(cudaMemsetAsync(t.buf->get(), 0, sizeof(S) * n, c.stream));
  }
  return t;
}

template <class S>
BTensor<S> clone(Ctx& c, const BTensor<S>& t) {
  BTensor<S> r;
  r.st = t.st;
  r.off = t.off;
  r.nelem = t.nelem;
  r.host = t.host;
  r.buf = std::make_shared<DevBuf>();
  if (t.nelem > 0) {
    r.buf->alloc(sizeof(S) * t.nelem, c.stream);
    SADMRG_CUDA(cudaMemcpyAsync(r.buf->get(), t.buf->get(), sizeof(S) * t.nelem, cudaMemcpyDeviceToDevice, c.stream));
  }
  return r;
}

// ---------------------------------------------------------------------------
// plan
int GemmPlan::add_job(int stage, int cbuf, long long coff, int m, int n, int ldc, int flags) {
  GemmJob j{};
  j.coff = coff; j.cbuf = cbuf; j.m = m; j.n = n; j.ldc = ldc; j.flags = flags;
  jobs.push_back(j);
  job_terms.emplace_back();
  job_stage.push_back(stage);
  return (int)jobs.size() - 1;
}

void GemmPlan::add_term(int job, int abuf, long long aoff, int lda, int bbuf, long long boff, int ldb, int k, int flags,
                        double ar, double ai) {
  GemmTerm t{};
  t.aoff = aoff; t.boff = boff; t.abuf = abuf; t.bbuf = bbuf;
  t.lda = std::max(lda, 1); t.ldb = std::max(ldb, 1); t.k = k; t.flags = flags; t.ar = ar; t.ai = ai;
  job_terms[job].push_back(t);
}

void GemmPlan::build_schedule(GemmSchedule& sc, bool cplx) {
  const int BM = sc.bm, BN = sc.bn;
  sc.items.clear();
  sc.reds.clear();
  sc.stage_items.assign(nstage + 1, 0);
  sc.stage_reds.assign(nstage + 1, 0);
  int nslot = 0;
  for (int s = 0; s < nstage; ++s) {
    // split-K chunk: enough items to fill the GPU, never below 128 of k
    long long total = 0;
    for (size_t j = 0; j < jobs.size(); ++j) {
      if (job_stage[j] != s) continue;
      long long kt = 0;
      for (auto& t : job_terms[j]) kt += t.k;
      total += (long long)((jobs[j].m + BM - 1) / BM) * ((jobs[j].n + BN - 1) / BN) * std::max<long long>(kt, 1);
    }
    long long ntile = 0;
    for (size_t j = 0; j < jobs.size(); ++j)
      if (job_stage[j] == s)
        ntile += (long long)((jobs[j].m + BM - 1) / BM) * ((jobs[j].n + BN - 1) / BN);
    // split the reduction only when the output tiles alone cannot fill the GPU
    long long kc = (total + target_items - 1) / std::max(target_items, 1);
    kc = std::max<long long>(128, (kc + 15) / 16 * 16);
    if (ntile >= target_items / 2) kc = (long long)1 << 40;
    std::vector<std::pair<long long, WorkItem>> its;
    for (size_t j = 0; j < jobs.size(); ++j) {
      if (job_stage[j] != s) continue;
      long long kt = 0;
      for (auto& t : job_terms[j]) kt += t.k;
      if (kt == 0 && (jobs[j].flags & JF_ACCUM)) continue;
      const int tm = (jobs[j].m + BM - 1) / BM, tn = (jobs[j].n + BN - 1) / BN;
      const long long nch = std::max<long long>(1, (kt + kc - 1) / kc);
      for (int a = 0; a < tm; ++a)
        for (int b = 0; b < tn; ++b) {
          if (nch == 1) {
            its.push_back({kt, WorkItem{(int)j, a, b, 0, 0, (int)kt, -1, -1}});
            continue;
          }
          const int slot0 = nslot, red = (int)sc.reds.size();
          long long pos = 0;
          int t = 0, k = 0;
          for (long long ch = 0; ch < nch; ++ch) {
            const long long len = std::min(kc, kt - pos);
            its.push_back({len, WorkItem{(int)j, a, b, t, k, (int)len, nslot++, red}});
            // advance (t, k) by len along the concatenated k
            long long left = len;
            while (left > 0) {
              const int avail = job_terms[j][t].k - k;
              if (left < avail) { k += (int)left; left = 0; }
              else { left -= avail; ++t; k = 0; }
            }
            pos += len;
          }
          sc.reds.push_back(RedItem{(int)j, a, b, slot0, (int)nch});
        }
    }
    // longest work first
    std::stable_sort(its.begin(), its.end(), [](const std::pair<long long, WorkItem>& x,
                                                const std::pair<long long, WorkItem>& y) { return x.first > y.first; });
    sc.stage_items[s] = (int)sc.items.size();
    for (auto& p : its) sc.items.push_back(p.second);
    sc.stage_items[s + 1] = (int)sc.items.size();
    sc.stage_reds[s + 1] = (int)sc.reds.size();
  }
  for (int s = 0; s < nstage; ++s) {
    sc.stage_items[s + 1] = std::max(sc.stage_items[s + 1], sc.stage_items[s]);
    sc.stage_reds[s + 1] = std::max(sc.stage_reds[s + 1], sc.stage_reds[s]);
  }
  sc.nslot = nslot;
  (void)cplx;
}

void GemmPlan::finalize(Ctx& c, bool cplx, bool mixed, const Bases* const_bases) {
  flat_terms.clear();
  flops = 0;
  for (size_t j = 0; j < jobs.size(); ++j) {
    jobs[j].t0 = (int)flat_terms.size();
    jobs[j].nt = (int)job_terms[j].size();
    for (auto& t : job_terms[j]) {
      flat_terms.push_back(t);
      flops += (cplx ? 8LL : 2LL) * jobs[j].m * (long long)jobs[j].n * t.k;
    }
  }
  sched = GemmSchedule{};
  sched.bm = gemm_tile_m(cplx, 0);
  sched.bn = gemm_tile_n(cplx, 0);
  build_schedule(sched, cplx);

  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t bt = sizeof(GemmTerm) * flat_terms.size(), bj = sizeof(GemmJob) * jobs.size(),
               bi = sizeof(WorkItem) * sched.items.size(), br = sizeof(RedItem) * sched.reds.size();
  const size_t total = al(bt) + al(bj) + al(bi) + al(br) + 256;
  std::vector<unsigned char> h(total, 0);
  if (bt) std::memcpy(h.data(), flat_terms.data(), bt);
  if (bj) std::memcpy(h.data() + al(bt), jobs.data(), bj);
  if (bi) std::memcpy(h.data() + al(bt) + al(bj), sched.items.data(), bi);
  if (br) std::memcpy(h.data() + al(bt) + al(bj) + al(bi), sched.reds.data(), br);
  dev = std::make_shared<DevBuf>(total, c.stream);
  SADMRG_CUDA(cudaMemcpyAsync(dev->get(), h.data(), total, cudaMemcpyHostToDevice, c.stream));
  unsigned char* base = dev->as<unsigned char>();
  d_terms = reinterpret_cast<GemmTerm*>(base);
  d_jobs = reinterpret_cast<GemmJob*>(base + al(bt));
  sched.d_items = reinterpret_cast<WorkItem*>(base + al(bt) + al(bj));
  sched.d_reds = reinterpret_cast<RedItem*>(base + al(bt) + al(bj) + al(bi));
  sched.work = std::make_shared<DevBuf>((size_t)std::max(sched.nslot, 1) * sched.bm * sched.bn * (cplx ? 16 : 8),
                                        c.stream);
  sched.tile_cnt = std::make_shared<DevBuf>(sizeof(int) * std::max<size_t>(sched.reds.size(), 1), c.stream);
  SADMRG_CUDA(cudaMemsetAsync(sched.tile_cnt->get(), 0, sched.tile_cnt->bytes(), c.stream));
  umma.reset();
  if (mixed && const_bases) {
    this->const_bases = *const_bases;
    build_umma(c, *const_bases, cplx);
  }
  // the host copies must stay alive until the async copies complete
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));
}

// tcgen05 schedule (see UmmaSchedule).  Returns false, leaving umma empty, when
// some term does not fit the panel scheme; the plan then runs 3xTF32 on the
// mma.sync kernels.
bool GemmPlan::build_umma(Ctx& c, const Bases& cb, bool cplx) {
  auto U = std::make_shared<UmmaSchedule>();
  const int nsm = device_sm_count();
  // tile width: 128 when the 128-wide output tiles alone fill the GPU twice per stage
  long long t128 = 0;
  for (size_t j = 0; j < jobs.size(); ++j)
    t128 += (long long)(((cplx ? 2 : 1) * jobs[j].m + 127) / 128) * ((jobs[j].n + 127) / 128);
  U->bn = tune.bn == 64 || tune.bn == 128 ? tune.bn : (t128 >= 2LL * nsm * std::max(nstage, 1)) ? 128 : 64;
  U->ctas = (tune.ctas == 2 && U->bn == 64) ? 2 : 1;
  const int BN = U->bn;

  struct Key {
    int buf;
    long long src;
    int ld, rows, K, trans, T;
    int cm;          // 2 * cmode + conj (PackJob)
    bool operator<(const Key& o) const {
      return std::tie(buf, src, ld, rows, K, trans, T, cm) <
             std::tie(o.buf, o.src, o.ld, o.rows, o.K, o.trans, o.T, o.cm);
    }
  };
  struct Pk {
    Key k;
    int cls;         // 0: constant (buffer 2), 1: psi (buffer 0), 2: stage-0 result (buffer 3)
    long long dst;
  };
  std::map<Key, int> index;
  std::vector<Pk> packs;
  auto get = [&](int buf, long long src, int ld, int rows, int K, int trans, int T, int cm) -> int {
    const Key k{buf, src, ld, rows, K, trans, T, cm};
    auto it = index.find(k);
    if (it != index.end()) return it->second;
    const int cls = buf == 2 ? 0 : buf == 0 ? 1 : buf == 3 ? 2 : -1;
    if (cls < 0) return -1;
    packs.push_back(Pk{k, cls, 0});
    index[k] = (int)packs.size() - 1;
    return (int)packs.size() - 1;
  };
  auto nslab_of = [](int K) { return (K + kPanelK - 1) / kPanelK; };
  auto panel_bytes = [&](const Key& k) {
    return (long long)((k.rows + k.T - 1) / k.T) * nslab_of(k.K) * k.T * 256;
  };
  std::vector<int> ta(flat_terms.size(), -1), tb(flat_terms.size(), -1);
  std::map<long long, double> xalpha;   // stage-0 result offset -> the one alpha its readers use
  for (size_t j = 0; j < jobs.size(); ++j) {
    const GemmJob& J = jobs[j];
    for (int t = J.t0; t < J.t0 + J.nt; ++t) {
      const GemmTerm& T = flat_terms[t];
      if (T.k == 0) continue;
      if (T.ai != 0.0) return false;
      // complex: Ah (2m x 2k, cmode 1) times Bh (2k x n, cmode 2)
      const int xm = cplx ? 2 : 1;
      const int cma = cplx ? 2 + ((T.flags & TF_CA) ? 1 : 0) : 0;
      const int cmb = cplx ? 4 + ((T.flags & TF_CB) ? 1 : 0) : 0;
      const int a = get(T.abuf, T.aoff, T.lda, xm * J.m, xm * T.k, (T.flags & TF_TA) ? 1 : 0, kUmmaTileM, cma);
      const int b = get(T.bbuf, T.boff, T.ldb, J.n, xm * T.k, (T.flags & TF_TB) ? 0 : 1, BN, cmb);
      if (a < 0 || b < 0 || packs[b].cls == 2) return false;
      if (packs[a].cls == 2) {
        if (T.flags & (TF_TA | TF_CA)) return false;
        auto it = xalpha.find(T.aoff);
        if (it == xalpha.end()) xalpha[T.aoff] = T.ar;
        else if (it->second != T.ar) return false;
      } else if (T.ar != 1.0) {
        return false;
      }
      ta[t] = a;
      tb[t] = b;
    }
  }
  long long cbytes = 0, vbytes = 0;
  for (auto& p : packs) {
    long long& tot = p.cls == 0 ? cbytes : vbytes;
    p.dst = tot;
    tot += (panel_bytes(p.k) + 255) & ~255LL;
  }
  std::vector<int> vpack_of(packs.size(), -1);
  for (size_t pi = 0; pi < packs.size(); ++pi) {
    auto& p = packs[pi];
    if (p.cls == 2) continue;
    if (p.cls == 1) vpack_of[pi] = (int)U->vpack.size();
    PackJob P{};
    P.src = p.k.src;
    P.dst = p.dst;
    P.srcbuf = p.k.buf;
    P.ld = p.k.ld;
    P.rows = p.k.rows;
    P.K = p.k.K;
    P.trans = p.k.trans;
    P.T = p.k.T;
    P.cmode = p.k.cm >> 1;
    P.conj = p.k.cm & 1;
    // psi (packed every matvec): only its real rows and k groups; the padding of its
    // panels is zeroed once below and never written
    P.sparse = p.cls == 1 ? 1 : 0;
    const long long nch = P.sparse ? (long long)P.rows * ((P.K + 3) / 4)
                                   : (long long)((P.rows + P.T - 1) / P.T) * P.T * nslab_of(P.K) * 8;
    long long& cc = p.cls == 0 ? U->cchunks : U->vchunks;
    auto& blk = p.cls == 0 ? U->cblk : U->vblk;
    auto& list = p.cls == 0 ? U->cpack : U->vpack;
    P.chunk0 = cc;
    const long long nb = (nch + 255) / 256;
    for (long long i = 0; i < nb; ++i) blk.push_back((int)list.size());
    cc += nb * 256;
    list.push_back(P);
  }
  SADMRG_REQUIRE(U->cchunks < (1LL << 31) && U->vchunks < (1LL << 31), SADMRG_ERR_LIMIT,
                 "tcgen05 schedule: operand panels too large for one pack launch");
  // dependency counters: [0, nv) psi pack jobs, then one per stage-0 result read as panels
  const int nv = (int)U->vpack.size();
  std::map<long long, int> xdep;   // stage-0 result offset -> its counter
  for (size_t pi = 0; pi < packs.size(); ++pi)
    if (packs[pi].cls == 2 && !xdep.count(packs[pi].k.src)) {
      const int d = nv + (int)xdep.size();
      xdep[packs[pi].k.src] = d;
    }
  auto dep_of = [&](int pi) -> int {
    if (packs[pi].cls == 1) return vpack_of[pi];
    if (packs[pi].cls == 2) return xdep[packs[pi].k.src];
    return -1;
  };
  U->terms.resize(flat_terms.size());
  for (size_t t = 0; t < flat_terms.size(); ++t) {
    UTerm u{};
    u.adep = u.bdep = -1;
    const int K = (cplx ? 2 : 1) * flat_terms[t].k;
    if (K > 0) {
      u.adep = dep_of(ta[t]);
      u.bdep = dep_of(tb[t]);
      u.a = packs[ta[t]].dst;
      u.b = packs[tb[t]].dst;
      u.abuf = packs[ta[t]].cls ? 1 : 0;
      u.bbuf = packs[tb[t]].cls ? 1 : 0;
      u.nslab = nslab_of(K);
      u.klast = K - (u.nslab - 1) * kPanelK;
    }
    U->terms[t] = u;
  }
  // jobs: stage-0 results become the A panels their readers use
  std::map<long long, int> xreader;   // stage-0 result offset -> its pack
  for (size_t i = 0; i < packs.size(); ++i)
    if (packs[i].cls == 2) {
      if (xreader.count(packs[i].k.src)) return false;
      xreader[packs[i].k.src] = (int)i;
    }
  int produced = 0;
  U->jobs.resize(jobs.size());
  for (size_t j = 0; j < jobs.size(); ++j) {
    const GemmJob& J = jobs[j];
    const int xm = cplx ? 2 : 1;   // complex: the real form of C (interleaved storage read as real)
    UJob u{};
    u.coff = xm * J.coff;
    u.pack = -1;
    u.alpha = 1.0;
    u.cbuf = J.cbuf;
    u.m = xm * J.m;
    u.n = J.n;
    u.ldc = xm * J.ldc;
    u.cx = cplx ? 1 : 0;
    u.flags = J.flags;
    u.t0 = J.t0;
    u.nt = J.nt;
    u.tag = J.tag;
    u.dep = -1;
    if (J.cbuf == 3) {
      auto it = xreader.find(J.coff);
      if (it == xreader.end() || job_stage[j] != 0 || (J.flags & JF_ACCUM)) return false;
      const Key& k = packs[it->second].k;
      if (k.rows != xm * J.m || k.K != xm * J.n || k.ld != J.ldc || k.trans != 0 || k.T != kUmmaTileM ||
          k.cm != (cplx ? 2 : 0))
        return false;
      u.pack = packs[it->second].dst;
      u.alpha = xalpha[J.coff];
      u.pack_nslab = nslab_of(xm * J.n);
      u.dep = xdep[J.coff];
      ++produced;
    } else if (J.cbuf != 1) {
      return false;
    }
    U->jobs[j] = u;
  }
  if (produced != (int)xreader.size()) return false;
  U->dep_target.assign(nv + xdep.size(), 0);
  for (int b : U->vblk) U->dep_target[b] += 256;              // chunks (padded) per psi job
  for (size_t j = 0; j < jobs.size(); ++j)
    if (U->jobs[j].dep >= 0)
      U->dep_target[U->jobs[j].dep] =
          ((U->jobs[j].m + kUmmaTileM - 1) / kUmmaTileM) * ((jobs[j].n + BN - 1) / BN);   // tiles of the result

  // slab-granular items, longest first; split the reduction only when the
  // output tiles cannot keep every SM busy
  const int target = 4 * nsm;
  U->stage_items.assign(nstage + 1, 0);
  U->stage_reds.assign(nstage + 1, 0);
  int nslot = 0;
  for (int s = 0; s < nstage; ++s) {
    long long total = 0, ntile = 0;
    for (size_t j = 0; j < jobs.size(); ++j) {
      if (job_stage[j] != s) continue;
      long long ns = 0;
      for (int t = jobs[j].t0; t < jobs[j].t0 + jobs[j].nt; ++t) ns += U->terms[t].nslab;
      const long long tiles = (long long)((U->jobs[j].m + kUmmaTileM - 1) / kUmmaTileM) * ((jobs[j].n + BN - 1) / BN);
      ntile += tiles;
      total += tiles * std::max<long long>(ns, 1);
    }
    // slabs per chunk: about one SM's share of the stage and never below 16 --
    // every split item pays for an FP32 partial tile and the fix-up, which at
    // 4 slabs per chunk cost more than the balance won (D=512: 99 -> 60 us)
    long long kc = std::max<long long>(std::max(tune.kc_min, 1), (total + nsm - 1) / nsm);
    if (ntile >= target / 2 || tune.kc_min <= 0) kc = (long long)1 << 40;
    if (tune.kc_max > 0) kc = std::min<long long>(kc, tune.kc_max);
    std::vector<std::pair<long long, UItem>> its;
    for (size_t j = 0; j < jobs.size(); ++j) {
      if (job_stage[j] != s) continue;
      const GemmJob& J = jobs[j];
      long long ns = 0;
      for (int t = J.t0; t < J.t0 + J.nt; ++t) ns += U->terms[t].nslab;
      if (ns == 0 && (J.flags & JF_ACCUM)) continue;
      const int tm = (U->jobs[j].m + kUmmaTileM - 1) / kUmmaTileM, tn = (J.n + BN - 1) / BN;
      const long long nch = std::max<long long>(1, (ns + kc - 1) / kc);
      for (int a = 0; a < tm; ++a)
        for (int b = 0; b < tn; ++b) {
          if (nch == 1) {
            its.push_back({ns, UItem{(int)j, a, b, J.t0, 0, (int)ns, -1, -1}});
            continue;
          }
          const int slot0 = nslot, red = (int)U->reds.size();
          long long pos = 0;
          int t = J.t0, s0 = 0;
          for (long long ch = 0; ch < nch; ++ch) {
            const long long len = std::min(kc, ns - pos);
            its.push_back({len, UItem{(int)j, a, b, t, s0, (int)len, nslot++, red}});
            long long left = len;
            while (left > 0) {
              const int avail = U->terms[t].nslab - s0;
              if (left < avail) { s0 += (int)left; left = 0; }
              else { left -= avail; ++t; s0 = 0; }
            }
            pos += len;
          }
          U->reds.push_back(URed{(int)j, a, b, slot0, (int)nch});
        }
    }
    std::stable_sort(its.begin(), its.end(),
                     [](const std::pair<long long, UItem>& x, const std::pair<long long, UItem>& y) {
                       return x.first > y.first;
                     });
    U->stage_items[s] = (int)U->items.size();
    for (auto& p : its) U->items.push_back(p.second);
    U->stage_items[s + 1] = (int)U->items.size();
    U->stage_reds[s + 1] = (int)U->reds.size();
  }
  for (int s = 0; s < nstage; ++s) {
    U->stage_items[s + 1] = std::max(U->stage_items[s + 1], U->stage_items[s]);
    U->stage_reds[s + 1] = std::max(U->stage_reds[s + 1], U->stage_reds[s]);
  }
  U->nslot = nslot;

  // device copies: [cpack | vpack | terms | jobs | items | reds | cblk | vblk]
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t b0 = sizeof(PackJob) * U->cpack.size(), b1 = sizeof(PackJob) * U->vpack.size(),
               b2 = sizeof(UTerm) * U->terms.size(), b3 = sizeof(UJob) * U->jobs.size(),
               b4 = sizeof(UItem) * U->items.size(), b5 = sizeof(URed) * U->reds.size(),
               b6 = sizeof(int) * U->cblk.size(), b7 = sizeof(int) * U->vblk.size(),
               b8 = sizeof(int) * U->dep_target.size();
  const size_t o1 = al(b0), o2 = o1 + al(b1), o3 = o2 + al(b2), o4 = o3 + al(b3), o5 = o4 + al(b4),
               o6 = o5 + al(b5), o7 = o6 + al(b6), o8 = o7 + al(b7), total = o8 + al(b8) + 256;
  std::vector<unsigned char> h(total, 0);
  if (b0) std::memcpy(h.data(), U->cpack.data(), b0);
  if (b1) std::memcpy(h.data() + o1, U->vpack.data(), b1);
  if (b2) std::memcpy(h.data() + o2, U->terms.data(), b2);
  if (b3) std::memcpy(h.data() + o3, U->jobs.data(), b3);
  if (b4) std::memcpy(h.data() + o4, U->items.data(), b4);
  if (b5) std::memcpy(h.data() + o5, U->reds.data(), b5);
  if (b6) std::memcpy(h.data() + o6, U->cblk.data(), b6);
  if (b7) std::memcpy(h.data() + o7, U->vblk.data(), b7);
  if (b8) std::memcpy(h.data() + o8, U->dep_target.data(), b8);
  U->dev = std::make_shared<DevBuf>(total, c.stream);
  SADMRG_CUDA(cudaMemcpyAsync(U->dev->get(), h.data(), total, cudaMemcpyHostToDevice, c.stream));
  unsigned char* base = U->dev->as<unsigned char>();
  const PackJob* d_cpack = reinterpret_cast<PackJob*>(base);
  U->d_vpack = reinterpret_cast<PackJob*>(base + o1);
  U->d_terms = reinterpret_cast<UTerm*>(base + o2);
  U->d_jobs = reinterpret_cast<UJob*>(base + o3);
  U->d_items = reinterpret_cast<UItem*>(base + o4);
  U->d_reds = reinterpret_cast<URed*>(base + o5);
  const int* d_cblk = reinterpret_cast<int*>(base + o6);
  U->d_vblk = reinterpret_cast<int*>(base + o7);
  U->d_dep_target = reinterpret_cast<int*>(base + o8);
  U->pconst = std::make_shared<DevBuf>((size_t)std::max<long long>(cbytes, 256), c.stream);
  U->pvar = std::make_shared<DevBuf>((size_t)std::max<long long>(vbytes, 256), c.stream);
  SADMRG_CUDA(cudaMemsetAsync(U->pvar->get(), 0, U->pvar->bytes(), c.stream));   // the padding of the psi panels
  U->slots = std::make_shared<DevBuf>((size_t)std::max(nslot, 1) * kUmmaTileM * BN * sizeof(float), c.stream);
  U->tile_cnt = std::make_shared<DevBuf>(sizeof(int) * std::max<size_t>(U->reds.size(), 1), c.stream);
  SADMRG_CUDA(cudaMemsetAsync(U->tile_cnt->get(), 0, U->tile_cnt->bytes(), c.stream));
  U->deps = std::make_shared<DevBuf>(sizeof(int) * (U->dep_target.size() + 1), c.stream);   // + fin
  SADMRG_CUDA(cudaMemsetAsync(U->deps->get(), 0, U->deps->bytes(), c.stream));
  launch_pack(d_cpack, d_cblk, (int)U->cblk.size(), cb, U->pconst->as<unsigned char>(), c.stream);
  ++c.launches;
  SADMRG_CUDA(cudaGetLastError());
  // the host image must outlive the async copy
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  umma = U;
  return true;
}

bool GemmPlan::rebuild_umma(Ctx& c, bool cplx) {
  if (!umma) return false;
  umma.reset();
  return build_umma(c, const_bases, cplx);
}

std::string GemmPlan::tune_key(bool cplx) const {
  auto lg = [](long long v) { int r = 0; while (v > 1) { v >>= 1; ++r; } return r; };
  std::map<std::tuple<int, int, int, int>, int> hist;
  for (size_t j = 0; j < jobs.size(); ++j) {
    long long kt = 0;
    for (auto& t : job_terms[j]) kt += t.k;
    ++hist[std::make_tuple(job_stage[j], lg(jobs[j].m), lg(jobs[j].n), lg(std::max<long long>(kt, 1)))];
  }
  std::string k = std::string(cplx ? "z" : "d") + std::to_string(device_sm_count()) + ":";
  for (auto& e : hist)
    k += std::to_string(std::get<0>(e.first)) + "," + std::to_string(std::get<1>(e.first)) + "," +
         std::to_string(std::get<2>(e.first)) + "," + std::to_string(std::get<3>(e.first)) + "x" +
         std::to_string(lg(e.second)) + ";";
  return k;
}

bool GemmPlan::runs_fused(const Ctx& c, bool cplx, int prec) const {
  if (!uses_umma(cplx, prec) || c.job_mask || (int)umma->vpack.size() > kMaxPackJobs) return false;
  if (tune.fused >= 0 && c.fused_matvec < 0) return tune.fused > 0;
  // small plans are latency bound and gain from one launch (D=512: 57 -> 46 us);
  // large ones lose to the dependency waits (D=2048: 494 -> 583 us)
  return c.fused_matvec > 0 || (c.fused_matvec < 0 && (double)flops < Ctx::kAutoFuseFlops);
}

int GemmPlan::launches_per_run(bool cplx, int prec, bool c_fused) const {
  int n = 0;
  if (uses_umma(cplx, prec)) {
    const UmmaSchedule& U = *umma;
    if (c_fused) return 1;   // pack + both stages in one launch
    int n = U.vblk.empty() ? 0 : 1;
    for (int s = 0; s < nstage; ++s)
      if (U.stage_items[s + 1] > U.stage_items[s]) ++n;
    return n;
  }
  for (int s = 0; s < nstage; ++s)
    if (sched.stage_items[s + 1] > sched.stage_items[s]) ++n;
  return n;
}

void GemmPlan::reset_counters(Ctx& c) const {
  if (sched.tile_cnt && sched.tile_cnt->bytes())
    SADMRG_CUDA(cudaMemsetAsync(sched.tile_cnt->get(), 0, sched.tile_cnt->bytes(), c.stream));
  if (umma) {
    if (umma->tile_cnt && umma->tile_cnt->bytes())
      SADMRG_CUDA(cudaMemsetAsync(umma->tile_cnt->get(), 0, umma->tile_cnt->bytes(), c.stream));
    if (umma->deps && umma->deps->bytes())   // the dependency counters and the finished-CTA count
      SADMRG_CUDA(cudaMemsetAsync(umma->deps->get(), 0, umma->deps->bytes(), c.stream));
  }
}

void GemmPlan::run_starved(Ctx& c, bool cplx, const Bases& b, int starve, long long wait_ns) const {
  SADMRG_REQUIRE(umma && !umma->vblk.empty() && starve >= 0 && starve < (int)umma->dep_target.size(),
                 SADMRG_ERR_STATE, "starved run: the plan has no tcgen05 schedule with psi panels");
  SADMRG_REQUIRE((int)umma->vpack.size() <= kMaxPackJobs, SADMRG_ERR_STATE, "starved run: too many pack jobs");
  const UmmaSchedule& U = *umma;
  std::vector<int> tgt = U.dep_target;
  tgt[starve] += 1;   // one more than the launch will ever count: nothing completes it
  DevBuf dt(sizeof(int) * tgt.size(), c.stream);
  SADMRG_CUDA(cudaMemcpyAsync(dt.get(), tgt.data(), sizeof(int) * tgt.size(), cudaMemcpyHostToDevice, c.stream));
  UBufs ub{};
  ub.pconst = U.pconst->as<unsigned char>();
  ub.pvar = U.pvar->as<unsigned char>();
  ub.slots = U.slots->as<float>();
  ub.tile_cnt = U.tile_cnt->as<int>();
  ub.deps = U.deps->as<int>();
  ub.dep_target = dt.as<int>();
  ub.fin = reinterpret_cast<unsigned*>(U.deps->as<int>() + U.dep_target.size());
  ub.mask = nullptr;
  UPhase ph{};
  ph.pk = U.d_vpack;
  ph.pk_blk = U.d_vblk;
  ph.npk_jobs = (int)U.vpack.size();
  ph.ndeps = (int)U.dep_target.size();
  ph.npk_blocks = (int)U.vblk.size();
  ph.wait_deps = 1;
  ph.wait_ns = wait_ns;
  ph.ctas_per_sm = U.ctas;
  const int ni = U.stage_items[nstage] - U.stage_items[0];
  launch_umma_items(U.bn, U.d_terms, U.d_jobs, U.d_items, U.d_reds, ni, b, ub, ph, c.stream);
  ++c.launches;
  SADMRG_CUDA(cudaGetLastError());
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));   // dt must outlive the launch
  (void)cplx;
}

static void mark(Ctx& c, int kind) {
  if (!c.prof) return;
  cudaEvent_t e;
  SADMRG_CUDA(cudaEventCreate(&e));
  SADMRG_CUDA(cudaEventRecord(e, c.stream));
  c.prof->push_back({kind, e});
}

void GemmPlan::run(Ctx& c, bool cplx, int prec, const Bases& b, int stage_lo, int stage_hi,
                   void* work_override) const {
  if (stage_hi < 0) stage_hi = nstage;
  if (uses_umma(cplx, prec)) {
    const UmmaSchedule& U = *umma;
    UBufs ub{};
    ub.pconst = U.pconst->as<unsigned char>();
    ub.pvar = U.pvar->as<unsigned char>();
    ub.slots = work_override ? static_cast<float*>(work_override) : U.slots->as<float>();
    ub.tile_cnt = U.tile_cnt->as<int>();
    ub.deps = U.deps->as<int>();
    ub.dep_target = U.d_dep_target;
    ub.fin = reinterpret_cast<unsigned*>(U.deps->as<int>() + U.dep_target.size());
    ub.mask = c.job_mask;
    UPhase ph{};
    ph.pk = U.d_vpack;
    ph.pk_blk = U.d_vblk;
    ph.npk_jobs = (int)U.vpack.size();
    ph.ndeps = (int)U.dep_target.size();
    ph.ctas_per_sm = U.ctas;
    const bool whole = stage_lo == 0 && stage_hi == nstage;
    if (whole && runs_fused(c, cplx, prec)) {
      // the whole matvec in one cooperative launch: psi packing, stage 0, stage 1
      ph.npk_blocks = (int)U.vblk.size();
      ph.wait_deps = 1;
      const int ni = U.stage_items[nstage] - U.stage_items[0];
      launch_umma_items(U.bn, U.d_terms, U.d_jobs, U.d_items, U.d_reds, ni, b, ub, ph, c.stream);
      ++c.launches;
      mark(c, 5);
    } else {
      if (stage_lo == 0 && !U.vblk.empty()) {
        launch_pack(U.d_vpack, U.d_vblk, (int)U.vblk.size(), b, ub.pvar, c.stream);
        ++c.launches;
        mark(c, 0);
      }
      for (int s = stage_lo; s < stage_hi; ++s) {
        const int ni = U.stage_items[s + 1] - U.stage_items[s];
        if (ni > 0) {
          launch_umma_items(U.bn, U.d_terms, U.d_jobs, U.d_items + U.stage_items[s], U.d_reds, ni, b, ub, ph,
                            c.stream);
          ++c.launches;
          mark(c, 1 + 2 * s);
        }
      }
    }
    SADMRG_CUDA(cudaGetLastError());
    c.gemm_flops += flops;
    return;
  }
  void* wk = work_override ? work_override : sched.work->get();
  for (int s = stage_lo; s < stage_hi; ++s) {
    const int ni = sched.stage_items[s + 1] - sched.stage_items[s];
    if (ni > 0) {
      launch_items(cplx, prec, d_terms, d_jobs, sched.d_items + sched.stage_items[s], ni, b, wk, sched.d_reds,
                   sched.tile_cnt->as<int>(), c.job_mask, c.stream);
      ++c.launches;
      mark(c, 1 + 2 * s);
    }
  }
  SADMRG_CUDA(cudaGetLastError());
  c.gemm_flops += flops;
}

namespace ops {

template <class S> static constexpr bool kC = ScalarInfo<S>::cplx;
template <class S> static double re_of(S x) { return real_of(x); }
static double im_of(double) { return 0.0; }
static double im_of(dcmplex x) { return x.imag(); }

static Struct mk(Sym s, int ls, std::vector<Bond> b) { return Struct(s, ls, std::move(b)); }

// Run a two-stage plan whose scratch products go to base 'sbuf'.
template <class S>
static void exec(Ctx& c, GemmPlan& p, Bases b, int sbuf) {
  if (p.empty()) return;
  p.finalize(c, kC<S>);
  DevBuf scratch;
  if (p.scratch_elems > 0) scratch.alloc(sizeof(S) * p.scratch_elems, c.stream);
  b.p[sbuf] = scratch.get();
  p.run(c, kC<S>, PREC_FP64, b);
}

// fuse(b1, b2): 3-leg identity embedding (src/block_tensor_inst.cpp:708-748)
template <class S>
BTensor<S> fuse(Ctx& c, const Bond& b1, const Bond& b2) {
  Bond f = Bond::fuse(c.sym, b1, b2);
  Struct st = mk(c.sym, 0, {b1, b2, f});
  const long nt = st.nten();
  std::vector<char> pres(nt, 0);
  int q[8], d[8];
  for (long i = 0; i < nt; ++i) pres[i] = st.block(i, q, d) ? 1 : 0;
  BTensor<S> t = alloc_tensor<S>(c, st, pres);
  std::vector<int> pos(f.nmom(), 0);
  std::vector<FuseFill> ff;
  for (long i = 0; i < nt; ++i) {
    if (!pres[i]) continue;
    st.block(i, q, d);
    const int k = f.index_of(q[2]);
    SADMRG_REQUIRE(pos[k] + d[0] * d[1] <= d[2], SADMRG_ERR_ARG, "fuse: fused dimension overflow");
    ff.push_back(FuseFill{t.off[i], d[0], d[1], d[2], pos[k]});
    pos[k] += d[0] * d[1];
  }
  if (!ff.empty()) {
    DevBuf dff(sizeof(FuseFill) * ff.size(), c.stream);
    SADMRG_CUDA(cudaMemcpyAsync(dff.get(), ff.data(), sizeof(FuseFill) * ff.size(), cudaMemcpyHostToDevice, c.stream));
    launch_fuse_fill(kC<S>, t.data(), dff.as<FuseFill>(), (int)ff.size(), c.stream);
    ++c.launches;
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  }
  return t;
}

// fuse_to_singlet: all-ones 2-leg blocks (src/block_tensor_inst.cpp:785-816)
template <class S>
BTensor<S> fuse_to_singlet(Ctx& c, const Bond& b1, const Bond& b2) {
  Struct st = mk(c.sym, 0, {b1, b2});
  const int n1 = b1.nmom(), n2 = b2.nmom();
  std::vector<char> pres(st.nten(), 0);
  for (int j = 0; j < n2; ++j)
    for (int i = 0; i < n1; ++i) {
      const bool ok = (c.sym == Sym::SU2) ? (b1.q[i] == b2.q[j]) : (b1.q[i] * b1.dir + b2.q[j] * b2.dir == 0);
      if (ok) pres[i + j * n1] = 1;
    }
  BTensor<S> t = alloc_tensor<S>(c, st, pres);
  launch_fill(kC<S>, t.data(), 1.0, 0.0, t.nelem, c.stream);
  ++c.launches;
  return t;
}

// overlap_initial (src/block_tensor_inst.cpp:1662-1788): out(a',b') = sum U^T conj(V)
template <class S>
BTensor<S> overlap_initial(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, int flag) {
  SADMRG_REQUIRE(uu.st.bonds[flag] == vv.st.bonds[flag] && uu.st.bonds[1 - flag] == vv.st.bonds[1 - flag],
                 SADMRG_ERR_ARG, "overlap_initial: inconsistent bonds");
  Bond b1 = vv.st.bonds[2];
  b1.invert();
  Struct st = mk(c.sym, 0, {uu.st.bonds[2], b1});
  auto U = blocks_of(uu), V = blocks_of(vv);
  std::vector<std::vector<std::pair<int, int>>> contrib(st.nten());
  for (size_t j = 0; j < U.size(); ++j)
    for (size_t k = 0; k < V.size(); ++k) {
      if (U[j].q[0] != V[k].q[0] || U[j].q[1] != V[k].q[1]) continue;
      int lab[2] = {U[j].q[2], V[k].q[2]};
      const long m = st.index(lab);
      SADMRG_REQUIRE(m >= 0, SADMRG_ERR_ARG, "overlap_initial: output sector missing");
      contrib[m].push_back({(int)j, (int)k});
    }
  std::vector<char> pres(st.nten(), 0);
  for (long m = 0; m < st.nten(); ++m) pres[m] = !contrib[m].empty();
  BTensor<S> out = alloc_tensor<S>(c, st, pres);
  GemmPlan p;
  for (long m = 0; m < st.nten(); ++m) {
    if (!pres[m]) continue;
    const Blk& u0 = U[contrib[m][0].first];
    const Blk& v0 = V[contrib[m][0].second];
    const int job = p.add_job(1, 2, out.off[m], u0.d[2], v0.d[2], u0.d[2], 0);
    for (auto& jk : contrib[m]) {
      const Blk& u = U[jk.first];
      const Blk& v = V[jk.second];
      const int k = u.d[0] * u.d[1];
      p.add_term(job, 0, u.off, k, 1, v.off, k, k, TF_TA | TF_CB, 1.0, 0.0);
    }
  }
  Bases b{};
  b.p[0] = uu.data(); b.p[1] = vv.data(); b.p[2] = out.data();
  exec<S>(c, p, b, 3);
  return out;
}

// overlap_transformation (src/block_tensor_inst.cpp:1791-1951): out = U^T op conj(V)
template <class S>
BTensor<S> overlap_transformation(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, const BTensor<S>& op, int flag) {
  {
    Bond a = op.st.bonds[0];
    a.invert();
    SADMRG_REQUIRE(uu.st.bonds[flag] == a && vv.st.bonds[flag] == op.st.bonds[1], SADMRG_ERR_ARG,
                   "overlap_transformation: inconsistent bonds");
  }
  Bond b1 = vv.st.bonds[2];
  b1.invert();
  Struct st = mk(c.sym, 0, {uu.st.bonds[2], b1});
  auto O = blocks_of(op), U = blocks_of(uu), V = blocks_of(vv);
  struct Item { int x; long long voff; int vrows; };
  std::vector<std::vector<Item>> contrib(st.nten());
  GemmPlan p;
  // stage 0: X = U^T op, once per (op block, uu block) pair that feeds an output
  for (size_t k = 0; k < U.size(); ++k)
    for (size_t j = 0; j < O.size(); ++j) {
      const Blk& o = O[j];
      const Blk& u = U[k];
      if (o.q[0] != u.q[flag]) continue;
      SADMRG_REQUIRE(u.d[1 - flag] == 1, SADMRG_ERR_ARG, "overlap_transformation: physical leg dim != 1");
      int x = -1;
      for (size_t l = 0; l < V.size(); ++l) {
        const Blk& v = V[l];
        if (o.q[1] != v.q[flag]) continue;
        if (u.q[1 - flag] != v.q[1 - flag]) continue;
        int lab[2] = {u.q[2], v.q[2]};
        if (!st.allowed_labels(lab)) continue;
        const long m = st.index(lab);
        if (x < 0) {
          const long long xo = p.alloc_scratch((long long)u.d[2] * o.d[1]);
          x = p.add_job(0, 3, xo, u.d[2], o.d[1], u.d[2], 0);
          p.add_term(x, 0, u.off, u.d[flag], 2, o.off, o.d[0], u.d[flag], TF_TA, 1.0, 0.0);
        }
        contrib[m].push_back(Item{x, v.off, v.d[flag]});
      }
    }
  std::vector<char> pres(st.nten(), 0);
  for (long m = 0; m < st.nten(); ++m) pres[m] = !contrib[m].empty();
  BTensor<S> out = alloc_tensor<S>(c, st, pres);
  for (long m = 0; m < st.nten(); ++m) {
    if (!pres[m]) continue;
    int lab[8], dd[8];
    st.block(m, lab, dd);
    const int job = p.add_job(1, 4, out.off[m], dd[0], dd[1], dd[0], 0);
    for (auto& it : contrib[m]) {
      const GemmJob& x = p.jobs[it.x];
      p.add_term(job, 3, x.coff, x.m, 1, it.voff, it.vrows, x.n, TF_CB, 1.0, 0.0);
    }
  }
  Bases b{};
  b.p[0] = uu.data(); b.p[1] = vv.data(); b.p[2] = op.data(); b.p[4] = out.data();
  exec<S>(c, p, b, 3);
  return out;
}

// operator_transformation (src/block_tensor_inst.cpp:1472-1658): out(a',c,b') = fac U^T op conj(V)
template <class S>
BTensor<S> operator_transformation(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, const BTensor<S>& op, int flag) {
  {
    Bond a = op.st.bonds[0];
    a.invert();
    SADMRG_REQUIRE(uu.st.bonds[flag] == a && vv.st.bonds[flag] == op.st.bonds[2], SADMRG_ERR_ARG,
                   "operator_transformation: inconsistent bonds");
  }
  Bond b2 = vv.st.bonds[2];
  b2.invert();
  Struct st = mk(c.sym, 0, {uu.st.bonds[2], op.st.bonds[1], b2});
  auto O = blocks_of(op), U = blocks_of(uu), V = blocks_of(vv);
  struct Item { int x; long long voff; int vrows; double fac; };
  std::vector<std::vector<Item>> contrib(st.nten());
  GemmPlan p;
  for (size_t k = 0; k < U.size(); ++k)
    for (size_t j = 0; j < O.size(); ++j) {
      const Blk& o = O[j];
      const Blk& u = U[k];
      if (o.q[0] != u.q[flag]) continue;
      SADMRG_REQUIRE(u.d[1 - flag] == 1 && o.d[1] == 1, SADMRG_ERR_ARG,
                     "operator_transformation: physical / channel leg dim != 1");
      int x = -1;
      for (size_t l = 0; l < V.size(); ++l) {
        const Blk& v = V[l];
        if (o.q[2] != v.q[flag]) continue;
        if (u.q[1 - flag] != v.q[1 - flag]) continue;
        int lab[3] = {u.q[2], o.q[1], v.q[2]};
        if (!st.allowed_labels(lab)) continue;
        const long m = st.index(lab);
        double fac = 1.0;
        if (c.sym == Sym::SU2) {
          fac = c.cgc->transformation(flag, u.q[2], o.q[1], v.q[2], u.q[flag], v.q[flag], u.q[1 - flag]);
          if (std::fabs(fac) < 1e-8) continue;
        }
        if (x < 0) {
          const long long xo = p.alloc_scratch((long long)u.d[2] * o.d[2]);
          x = p.add_job(0, 3, xo, u.d[2], o.d[2], u.d[2], 0);
          p.add_term(x, 0, u.off, u.d[flag], 2, o.off, o.d[0], u.d[flag], TF_TA, 1.0, 0.0);
        }
        contrib[m].push_back(Item{x, v.off, v.d[flag], fac});
      }
    }
  std::vector<char> pres(st.nten(), 0);
  for (long m = 0; m < st.nten(); ++m) pres[m] = !contrib[m].empty();
  BTensor<S> out = alloc_tensor<S>(c, st, pres);
  for (long m = 0; m < st.nten(); ++m) {
    if (!pres[m]) continue;
    int lab[8], dd[8];
    st.block(m, lab, dd);
    const int job = p.add_job(1, 4, out.off[m], dd[0], dd[2], dd[0] * dd[1], 0);
    for (auto& it : contrib[m]) {
      const GemmJob& x = p.jobs[it.x];
      p.add_term(job, 3, x.coff, x.m, 1, it.voff, it.vrows, x.n, TF_CB, it.fac, 0.0);
    }
  }
  Bases b{};
  b.p[0] = uu.data(); b.p[1] = vv.data(); b.p[2] = op.data(); b.p[4] = out.data();
  exec<S>(c, p, b, 3);
  return out;
}

// operator_pairup (src/block_tensor_inst.cpp:1954-2167): out(a',b') = fac op2 U^T op1 conj(V)
template <class S>
BTensor<S> operator_pairup(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, const BTensor<S>& op1,
                           const BTensor<S>& op2, int flag) {
  {
    Bond a = op1.st.bonds[0];
    a.invert();
    Bond ch = op2.st.bonds[1];
    if (c.sym == Sym::U1) ch.invert();
    SADMRG_REQUIRE(uu.st.bonds[flag] == a && vv.st.bonds[flag] == op1.st.bonds[2] && op1.st.bonds[1] == ch,
                   SADMRG_ERR_ARG, "operator_pairup: inconsistent bonds");
    SADMRG_REQUIRE(!op2.host.empty(), SADMRG_ERR_STATE, "operator_pairup: site operator has no host copy");
  }
  Bond b1 = vv.st.bonds[2];
  b1.invert();
  Struct st = mk(c.sym, 0, {uu.st.bonds[2], b1});
  auto O = blocks_of(op1), U = blocks_of(uu), V = blocks_of(vv);
  // site operator blocks, including null ones (presence checked after matching)
  struct SBlk { int q[3]; long long off; };
  std::vector<SBlk> P;
  {
    int q[8], d[8];
    for (long n = 0; n < op2.nten(); ++n)
      if (op2.st.block(n, q, d)) P.push_back(SBlk{{q[0], q[1], q[2]}, op2.off[n]});
  }
  struct Item { int x; long long voff; int vrows; S alpha; };
  std::vector<std::vector<Item>> contrib(st.nten());
  GemmPlan p;
  for (size_t k = 0; k < U.size(); ++k)
    for (size_t j = 0; j < O.size(); ++j) {
      const Blk& o = O[j];
      const Blk& u = U[k];
      if (o.q[0] != u.q[flag]) continue;
      SADMRG_REQUIRE(u.d[1 - flag] == 1 && o.d[1] == 1, SADMRG_ERR_ARG, "operator_pairup: leg dim != 1");
      int x = -1;
      for (size_t l = 0; l < V.size(); ++l) {
        const Blk& v = V[l];
        if (o.q[2] != v.q[flag]) continue;
        for (auto& s2 : P) {
          if (s2.q[0] != u.q[1 - flag] || s2.q[2] != v.q[1 - flag] || s2.q[1] != o.q[1]) continue;
          int lab[2] = {u.q[2], v.q[2]};
          if (!st.allowed_labels(lab)) continue;
          const long m = st.index(lab);
          if (s2.off < 0) continue;
          double fac = 1.0;
          if (c.sym == Sym::SU2) {
            fac = c.cgc->pairup(flag, u.q[2], u.q[flag], v.q[flag], o.q[1], s2.q[0], s2.q[2]);
            if (std::fabs(fac) < 1e-8) continue;
          }
          if (x < 0) {
            const long long xo = p.alloc_scratch((long long)u.d[2] * o.d[2]);
            x = p.add_job(0, 3, xo, u.d[2], o.d[2], u.d[2], 0);
            p.add_term(x, 0, u.off, u.d[flag], 2, o.off, o.d[0], u.d[flag], TF_TA, 1.0, 0.0);
          }
          const S alpha = S(fac) * op2.host[s2.off];
          contrib[m].push_back(Item{x, v.off, v.d[flag], alpha});
        }
      }
    }
  std::vector<char> pres(st.nten(), 0);
  for (long m = 0; m < st.nten(); ++m) pres[m] = !contrib[m].empty();
  BTensor<S> out = alloc_tensor<S>(c, st, pres);
  for (long m = 0; m < st.nten(); ++m) {
    if (!pres[m]) continue;
    int lab[8], dd[8];
    st.block(m, lab, dd);
    const int job = p.add_job(1, 4, out.off[m], dd[0], dd[1], dd[0], 0);
    for (auto& it : contrib[m]) {
      const GemmJob& x = p.jobs[it.x];
      p.add_term(job, 3, x.coff, x.m, 1, it.voff, it.vrows, x.n, TF_CB, re_of(it.alpha), im_of(it.alpha));
    }
  }
  Bases b{};
  b.p[0] = uu.data(); b.p[1] = vv.data(); b.p[2] = op1.data(); b.p[4] = out.data();
  exec<S>(c, p, b, 3);
  return out;
}

// operator_initial (src/block_tensor_inst.cpp:1283-1469): out(a',c,b') = fac op U^T conj(V)
template <class S>
BTensor<S> operator_initial(Ctx& c, const BTensor<S>& uu, const BTensor<S>& vv, const BTensor<S>& op, int flag) {
  {
    Bond a = op.st.bonds[0];
    a.invert();
    SADMRG_REQUIRE(uu.st.bonds[1 - flag] == a && vv.st.bonds[1 - flag] == op.st.bonds[2], SADMRG_ERR_ARG,
                   "operator_initial: inconsistent bonds");
    SADMRG_REQUIRE(!op.host.empty(), SADMRG_ERR_STATE, "operator_initial: site operator has no host copy");
  }
  Bond b2 = vv.st.bonds[2];
  b2.invert();
  Struct st = mk(c.sym, 0, {uu.st.bonds[2], op.st.bonds[1], b2});
  auto O = blocks_of(op), U = blocks_of(uu), V = blocks_of(vv);
  struct Item { long long uoff, voff; int k; S alpha; };
  std::vector<std::vector<Item>> contrib(st.nten());
  for (size_t k = 0; k < U.size(); ++k)
    for (size_t j = 0; j < O.size(); ++j) {
      const Blk& o = O[j];
      const Blk& u = U[k];
      if (o.q[0] != u.q[1 - flag]) continue;
      SADMRG_REQUIRE(o.d[0] * o.d[1] * o.d[2] == 1, SADMRG_ERR_ARG, "operator_initial: site operator block not 1x1x1");
      for (size_t l = 0; l < V.size(); ++l) {
        const Blk& v = V[l];
        if (o.q[2] != v.q[1 - flag]) continue;
        if (u.q[flag] != v.q[flag]) continue;
        int lab[3] = {u.q[2], o.q[1], v.q[2]};
        if (!st.allowed_labels(lab)) continue;
        const long m = st.index(lab);
        double fac = 1.0;
        if (c.sym == Sym::SU2) {
          fac = c.cgc->onsite(flag, u.q[2], o.q[1], v.q[2], u.q[flag], o.q[0], o.q[2]);
          if (std::fabs(fac) < 1e-8) continue;
        }
        contrib[m].push_back(Item{u.off, v.off, u.d[0] * u.d[1], S(fac) * op.host[o.off]});
      }
    }
  std::vector<char> pres(st.nten(), 0);
  for (long m = 0; m < st.nten(); ++m) pres[m] = !contrib[m].empty();
  BTensor<S> out = alloc_tensor<S>(c, st, pres);
  GemmPlan p;
  for (long m = 0; m < st.nten(); ++m) {
    if (!pres[m]) continue;
    int lab[8], dd[8];
    st.block(m, lab, dd);
    const int job = p.add_job(1, 2, out.off[m], dd[0], dd[2], dd[0] * dd[1], 0);
    for (auto& it : contrib[m])
      p.add_term(job, 0, it.uoff, it.k, 1, it.voff, it.k, it.k, TF_TA | TF_CB, re_of(it.alpha), im_of(it.alpha));
  }
  Bases b{};
  b.p[0] = uu.data(); b.p[1] = vv.data(); b.p[2] = out.data();
  exec<S>(c, p, b, 3);
  return out;
}

// generic contraction (src/block_tensor_inst.cpp:1046-1126) for a contracted
// bond that is the first or the last of each operand (the shapes the sweep uses).
template <class S>
BTensor<S> contract(Ctx& c, const BTensor<S>& t1, int i1, const BTensor<S>& t2, int i2) {
  const int n1 = t1.st.nbond(), n2 = t2.st.nbond();
  SADMRG_REQUIRE((i1 == 0 || i1 == n1 - 1) && (i2 == 0 || i2 == n2 - 1), SADMRG_ERR_ARG,
                 "contract: contracted bond must be first or last");
  {
    Bond b = t2.st.bonds[i2];
    b.invert();
    SADMRG_REQUIRE(t1.st.bonds[i1] == b, SADMRG_ERR_ARG, "contract: bonds cannot be contracted");
  }
  std::vector<Bond> bb;
  for (int i = 0; i < n1 - 1; ++i) bb.push_back(t1.st.bonds[(i1 + 1 + i) % n1]);
  for (int i = 0; i < n2 - 1; ++i) bb.push_back(t2.st.bonds[(i2 + 1 + i) % n2]);
  Struct st = mk(c.sym, t1.st.locspin + t2.st.locspin, bb);
  const Bond& cb = t1.st.bonds[i1];
  struct Item { long long aoff, boff; int k; };
  std::vector<std::vector<Item>> contrib(st.nten());
  std::vector<int> rowsA(st.nten(), 0), colsB(st.nten(), 0);
  int q[8], d[8], qa[8], qb[8];
  for (long m = 0; m < st.nten(); ++m) {
    if (!st.block(m, q, d)) continue;
    for (int k = 0; k < n1 - 1; ++k) qa[(i1 + 1 + k) % n1] = q[k];
    for (int k = 0; k < n2 - 1; ++k) qb[(i2 + 1 + k) % n2] = q[k + n1 - 1];
    for (int j = 0; j < cb.nmom(); ++j) {
      qa[i1] = cb.q[j];
      qb[i2] = cb.q[j];
      if (!t1.st.allowed_labels(qa) || !t2.st.allowed_labels(qb)) continue;
      const long ka = t1.st.index(qa), kb = t2.st.index(qb);
      if (ka < 0 || kb < 0 || !t1.present(ka) || !t2.present(kb)) continue;
      contrib[m].push_back(Item{t1.off[ka], t2.off[kb], cb.d[j]});
    }
  }
  std::vector<char> pres(st.nten(), 0);
  for (long m = 0; m < st.nten(); ++m) pres[m] = !contrib[m].empty();
  BTensor<S> out = alloc_tensor<S>(c, st, pres);
  GemmPlan p;
  for (long m = 0; m < st.nten(); ++m) {
    if (!pres[m]) continue;
    st.block(m, q, d);
    long long rows = 1, cols = 1;
    for (int k = 0; k < n1 - 1; ++k) rows *= d[k];
    for (int k = 0; k < n2 - 1; ++k) cols *= d[n1 - 1 + k];
    const int job = p.add_job(1, 2, out.off[m], (int)rows, (int)cols, (int)rows, 0);
    for (auto& it : contrib[m]) {
      // A' = t1 with the contracted bond last (rows x k): transposed view when it is first
      const int fa = (i1 == 0) ? TF_TA : 0;
      const int lda = (i1 == 0) ? it.k : (int)rows;
      const int fb = (i2 == 0) ? 0 : TF_TB;
      const int ldb = (i2 == 0) ? it.k : (int)cols;
      p.add_term(job, 0, it.aoff, lda, 1, it.boff, ldb, it.k, fa | fb, 1.0, 0.0);
    }
  }
  Bases b{};
  b.p[0] = t1.data(); b.p[1] = t2.data(); b.p[2] = out.data();
  exec<S>(c, p, b, 3);
  return out;
}

// dst += alpha_b * src block by block (BlockTensor::operator+= presence rules,
// src/block_tensor_inst.cpp:225-252); alpha_b = alpha, or alpha * chan_w[(q + 2) / 2]
// with q the U(1) charge of the block's channel leg (bond 1) when chan_w is given.
template <class S>
static void add_into_impl(Ctx& c, BTensor<S>& dst, const BTensor<S>& src, S alpha, const S* chan_w) {
  if (src.null()) return;
  if (dst.null()) {
    if (!chan_w) {
      dst = clone(c, src);
      if (alpha != S(1)) scale(c, dst, alpha);
      return;
    }
    std::vector<char> pres(src.nten(), 0);
    for (long i = 0; i < src.nten(); ++i) pres[i] = src.present(i);
    dst = alloc_tensor<S>(c, src.st, pres);   // zero-filled
  }
  SADMRG_REQUIRE(dst.st == src.st, SADMRG_ERR_ARG, "add_into: different structures");
  bool same = true;
  for (long i = 0; i < dst.nten(); ++i)
    if (src.present(i) && !dst.present(i)) { same = false; break; }
  BTensor<S> target;
  std::vector<Seg> sd, ss;
  if (!same) {
    std::vector<char> pres(dst.nten(), 0);
    for (long i = 0; i < dst.nten(); ++i) pres[i] = dst.present(i) || src.present(i);
    target = alloc_tensor<S>(c, dst.st, pres);
    for (long i = 0; i < dst.nten(); ++i)
      if (dst.present(i)) sd.push_back(Seg{target.off[i], dst.off[i], dst.st.block_elems(i), 1.0, 0.0});
  }
  BTensor<S>& T = same ? dst : target;
  int q[8], d[8];
  for (long i = 0; i < src.nten(); ++i) {
    if (!src.present(i)) continue;
    S a = alpha;
    if (chan_w) {
      src.st.block(i, q, d);
      const int ci = (q[1] + 2) / 2;
      SADMRG_REQUIRE(ci >= 0 && ci < 3 && q[1] % 2 == 0, SADMRG_ERR_ARG, "add_into: channel charge outside {-2,0,2}");
      a = alpha * chan_w[ci];
    }
    ss.push_back(Seg{T.off[i], src.off[i], src.st.block_elems(i), re_of(a), im_of(a)});
  }
  DevBuf dsegs(sizeof(Seg) * (sd.size() + ss.size()) + 16, c.stream);
  std::vector<Seg> all = sd;
  all.insert(all.end(), ss.begin(), ss.end());
  SADMRG_CUDA(cudaMemcpyAsync(dsegs.get(), all.data(), sizeof(Seg) * all.size(), cudaMemcpyHostToDevice, c.stream));
  if (!sd.empty()) { launch_seg_axpy(kC<S>, T.data(), dst.data(), dsegs.as<Seg>(), (int)sd.size(), c.stream); ++c.launches; }
  if (!ss.empty()) {
    launch_seg_axpy(kC<S>, T.data(), src.data(), dsegs.as<Seg>() + sd.size(), (int)ss.size(), c.stream);
    ++c.launches;
  }
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  if (!same) dst = std::move(target);
}

template <class S>
void add_into(Ctx& c, BTensor<S>& dst, const BTensor<S>& src, S alpha) {
  add_into_impl<S>(c, dst, src, alpha, nullptr);
}

template <class S>
void add_into_channels(Ctx& c, BTensor<S>& dst, const BTensor<S>& src, const S chan_w[3]) {
  SADMRG_REQUIRE(c.sym == Sym::U1, SADMRG_ERR_ARG, "add_into_channels: U(1) operators only");
  add_into_impl<S>(c, dst, src, S(1), chan_w);
}

template <class S>
void scale(Ctx& c, BTensor<S>& t, S alpha) {
  launch_scale(kC<S>, t.data(), re_of(alpha), im_of(alpha), t.nelem, c.stream);
  ++c.launches;
  if (!t.host.empty())
    for (auto& x : t.host) x *= alpha;
}

template <class S>
void take_conjugate(BTensor<S>& t, int bond) {
  t.st.bonds[bond].invert();
}

// makeup_input_vector (src/block_tensor_inst.cpp:1231-1257)
template <class S>
void makeup_input_vector(Ctx& c, BTensor<S>& t) {
  SADMRG_REQUIRE(t.st.nbond() == 2, SADMRG_ERR_ARG, "makeup_input_vector: not a 2-leg tensor");
  const Bond &b0 = t.st.bonds[0], &b1 = t.st.bonds[1];
  std::vector<char> pres(t.nten(), 0);
  bool changed = false;
  for (long i = 0; i < t.nten(); ++i) pres[i] = t.present(i);
  for (int i = 0; i < b0.nmom(); ++i)
    for (int j = 0; j < b1.nmom(); ++j)
      if (b0.q[i] == b1.q[j] && !pres[i + (long)j * b0.nmom()]) { pres[i + (long)j * b0.nmom()] = 1; changed = true; }
  if (!changed) return;
  BTensor<S> n = alloc_tensor<S>(c, t.st, pres);
  std::vector<Seg> sg;
  for (long i = 0; i < t.nten(); ++i)
    if (t.present(i)) sg.push_back(Seg{n.off[i], t.off[i], t.st.block_elems(i), 1.0, 0.0});
  if (!sg.empty()) {
    DevBuf d(sizeof(Seg) * sg.size(), c.stream);
    SADMRG_CUDA(cudaMemcpyAsync(d.get(), sg.data(), sizeof(Seg) * sg.size(), cudaMemcpyHostToDevice, c.stream));
    launch_seg_axpy(kC<S>, n.data(), t.data(), d.as<Seg>(), (int)sg.size(), c.stream);
    ++c.launches;
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  }
  t = std::move(n);
}

// left2right_vectran / right2left_vectran (src/block_tensor_inst.cpp:429-497)
template <class S>
static void vectran(Ctx& c, BTensor<S>& t, int ishift, int s0, int s1) {
  SADMRG_REQUIRE(t.st.nbond() == 3, SADMRG_ERR_ARG, "vectran: not a 3-leg tensor");
  Struct st1 = t.st.shifted(s0, s1);
  std::vector<char> pres(st1.nten(), 0);
  std::vector<std::pair<long, long>> map;
  int q[8], d[8], q1[8];
  for (long i = 0; i < t.nten(); ++i) {
    if (!t.st.block(i, q, d) || !t.present(i)) continue;
    for (int k = 0; k < 3; ++k) q1[(k + ishift) % 3] = q[k];
    const long j = st1.index(q1);
    if (j < 0) continue;
    pres[j] = 1;
    map.push_back({i, j});
  }
  if (c.sym == Sym::SU2) {
    st1.bonds[0].dir = 1;
    st1.bonds[1].dir = 1;
    st1.bonds[2].dir = -1;
  }
  BTensor<S> n = alloc_tensor<S>(c, st1, pres);
  std::vector<Transp> tr;
  for (auto& ij : map) {
    t.st.block(ij.first, q, d);
    // Dense::shift(s0, s1): transpose of (B x A) with B = product of the first p = 3 - ishift dims
    const int p = 3 - ishift;
    long long B = 1, A = 1;
    for (int k = 0; k < p; ++k) B *= d[k];
    for (int k = p; k < 3; ++k) A *= d[k];
    tr.push_back(Transp{t.off[ij.first], n.off[ij.second], (int)B, (int)A});
  }
  if (!tr.empty()) {
    DevBuf dt(sizeof(Transp) * tr.size(), c.stream);
    SADMRG_CUDA(cudaMemcpyAsync(dt.get(), tr.data(), sizeof(Transp) * tr.size(), cudaMemcpyHostToDevice, c.stream));
    launch_block_transpose(kC<S>, n.data(), t.data(), dt.as<Transp>(), (int)tr.size(), c.stream);
    ++c.launches;
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  }
  t = std::move(n);
}

template <class S> void left2right_vectran(Ctx& c, BTensor<S>& t) { vectran(c, t, 2, 1, 0); }
template <class S> void right2left_vectran(Ctx& c, BTensor<S>& t) { vectran(c, t, 1, 2, 0); }

// leg permutation of a 3-leg tensor (BlockTensor::shift / exchangeindex,
// src/block_tensor_inst.cpp:913-990, SU2Struct::shift src/symmetry/su2.cpp:509-518):
// the bonds move with their directions, a block keeps its presence under its
// permuted labels and its data is permuted on the device; for SU(2) the
// reference moves the CGC blocks along, which here the permuted bonds imply.
template <class S>
BTensor<S> permute3(Ctx& c, const BTensor<S>& t, const int p[3]) {
  SADMRG_REQUIRE(t.st.nbond() == 3, SADMRG_ERR_ARG, "permute3: a 3-leg tensor");
  std::vector<Bond> nb(3);
  for (int k = 0; k < 3; ++k) nb[k] = t.st.bonds[p[k]];
  Struct nst(c.sym, t.st.locspin, nb);
  std::vector<char> pres(nst.nten(), 0);
  std::vector<std::pair<long, long>> map;
  int q[8], d[8];
  for (long i = 0; i < t.nten(); ++i) {
    if (!t.present(i) || !t.st.block(i, q, d)) continue;
    const int nq[3] = {q[p[0]], q[p[1]], q[p[2]]};
    const long j = nst.index(nq);
    SADMRG_REQUIRE(j >= 0 && nst.allowed_labels(nq), SADMRG_ERR_STATE, "permute3: a block without a place");
    pres[j] = 1;
    map.push_back({i, j});
  }
  BTensor<S> n = alloc_tensor<S>(c, nst, pres);
  std::vector<Perm3> jobs;
  for (auto& ij : map) {
    t.st.block(ij.first, q, d);
    Perm3 J{};
    J.soff = t.off[ij.first];
    J.doff = n.off[ij.second];
    for (int k = 0; k < 3; ++k) { J.d[k] = d[k]; J.p[k] = p[k]; }
    jobs.push_back(J);
  }
  if (!jobs.empty()) {
    DevBuf dj(sizeof(Perm3) * jobs.size(), c.stream);
    SADMRG_CUDA(cudaMemcpyAsync(dj.get(), jobs.data(), sizeof(Perm3) * jobs.size(), cudaMemcpyHostToDevice, c.stream));
    launch_permute3(kC<S>, n.data(), t.data(), dj.as<Perm3>(), (int)jobs.size(), c.stream);
    ++c.launches;
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  }
  return n;
}

template <class S>
BTensor<S> from_host(Ctx& c, const Struct& st, const std::vector<char>& present, const S* data) {
  BTensor<S> t = alloc_tensor<S>(c, st, present);
  if (t.nelem > 0 && data)
    SADMRG_CUDA(cudaMemcpyAsync(t.data(), data, sizeof(S) * t.nelem, cudaMemcpyHostToDevice, c.stream));
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  return t;
}

template <class S>
std::vector<S> to_host(Ctx& c, const BTensor<S>& t) {
  std::vector<S> h(t.nelem);
  if (t.nelem > 0)
    SADMRG_CUDA(cudaMemcpyAsync(h.data(), t.data(), sizeof(S) * t.nelem, cudaMemcpyDeviceToHost, c.stream));
  SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  return h;
}

#define SADMRG_INST(S)                                                                                           \
  template BTensor<S> fuse<S>(Ctx&, const Bond&, const Bond&);                                                   \
  template BTensor<S> fuse_to_singlet<S>(Ctx&, const Bond&, const Bond&);                                        \
  template BTensor<S> overlap_initial<S>(Ctx&, const BTensor<S>&, const BTensor<S>&, int);                       \
  template BTensor<S> overlap_transformation<S>(Ctx&, const BTensor<S>&, const BTensor<S>&, const BTensor<S>&,   \
                                                int);                                                            \
  template BTensor<S> operator_initial<S>(Ctx&, const BTensor<S>&, const BTensor<S>&, const BTensor<S>&, int);   \
  template BTensor<S> operator_transformation<S>(Ctx&, const BTensor<S>&, const BTensor<S>&, const BTensor<S>&,  \
                                                 int);                                                           \
  template BTensor<S> operator_pairup<S>(Ctx&, const BTensor<S>&, const BTensor<S>&, const BTensor<S>&,          \
                                         const BTensor<S>&, int);                                                \
  template BTensor<S> contract<S>(Ctx&, const BTensor<S>&, int, const BTensor<S>&, int);                         \
  template void add_into<S>(Ctx&, BTensor<S>&, const BTensor<S>&, S);                                            \
  template void add_into_channels<S>(Ctx&, BTensor<S>&, const BTensor<S>&, const S*);                            \
  template void scale<S>(Ctx&, BTensor<S>&, S);                                                                  \
  template void take_conjugate<S>(BTensor<S>&, int);                                                             \
  template void makeup_input_vector<S>(Ctx&, BTensor<S>&);                                                       \
  template void left2right_vectran<S>(Ctx&, BTensor<S>&);                                                        \
  template void right2left_vectran<S>(Ctx&, BTensor<S>&);                                                        \
  template BTensor<S> permute3<S>(Ctx&, const BTensor<S>&, const int*);                                          \
  template BTensor<S> from_host<S>(Ctx&, const Struct&, const std::vector<char>&, const S*);                     \
  template std::vector<S> to_host<S>(Ctx&, const BTensor<S>&);

SADMRG_INST(double)
SADMRG_INST(dcmplex)

}  // namespace ops

template std::vector<Blk> blocks_of<double>(const BTensor<double>&);
template std::vector<Blk> blocks_of<dcmplex>(const BTensor<dcmplex>&);
template BTensor<double> alloc_tensor<double>(Ctx&, const Struct&, const std::vector<char>&);
template BTensor<dcmplex> alloc_tensor<dcmplex>(Ctx&, const Struct&, const std::vector<char>&);
template BTensor<double> clone<double>(Ctx&, const BTensor<double>&);
template BTensor<dcmplex> clone<dcmplex>(Ctx&, const BTensor<dcmplex>&);

}  // namespace sadmrg
