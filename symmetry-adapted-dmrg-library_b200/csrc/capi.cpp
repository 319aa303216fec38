// capi.cpp -- extern "C" boundary (include/sadmrg.h).
#include <cstring>
#include <memory>
#include <string>

#include "../../include/sadmrg.h"
#include "dmrg.hpp"

using namespace sadmrg;

template <class S>
struct State {
  std::unique_ptr<HeffPlan<S>> heff;
  std::unique_ptr<Chain<S>> chain;
  std::unique_ptr<HeffBatch<S>> batch;
  BTensor<S> staged[2];
  DevBuf io;   // psi in / out for host-buffer calls
};

struct sadmrg_handle {
  Ctx ctx;
  int device = 0;
  std::string err;
  State<double> sd;
  State<dcmplex> sz;
};

static int fail(sadmrg_handle* h, int code, const std::string& m) {
  if (h) h->err = m;
  return code;
}

template <class F>
static int guard(sadmrg_handle* h, F&& f) {
  if (!h) return SADMRG_ERR_ARG;
  try {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return fail(h, SADMRG_ERR_CUDA, cudaGetErrorString(e));
    f();
    return SADMRG_OK;
  } catch (const Error& e) {
    return fail(h, e.code, e.what());
  } catch (const std::exception& e) {
    return fail(h, SADMRG_ERR_ARG, e.what());
  }
}

template <class S>
static BTensor<S> from_desc(Ctx& c, const sadmrg_tensor_desc* t) {
  SADMRG_REQUIRE(t && t->nbond >= 1 && t->nbond <= 4, SADMRG_ERR_ARG, "tensor desc: bad nbond");
  std::vector<Bond> bonds;
  int o = 0;
  for (int b = 0; b < t->nbond; ++b) {
    std::vector<int> q(t->q + o, t->q + o + t->nmom[b]), d(t->d + o, t->d + o + t->nmom[b]);
    o += t->nmom[b];
    Bond bd;
    bd.dir = t->dir[b];
    bd.q = q;   // the caller gives the sectors in the reference's (sorted) order
    bd.d = d;
    for (size_t k = 1; k < q.size(); ++k)
      SADMRG_REQUIRE(q[k] > q[k - 1], SADMRG_ERR_ARG, "tensor desc: sector labels must ascend");
    bonds.push_back(bd);
  }
  Struct st(c.sym, t->locspin, bonds);
  std::vector<char> pres(st.nten(), 0);
  for (int i = 0; i < t->nblocks; ++i) {
    const long long bi = t->block_index[i];
    SADMRG_REQUIRE(bi >= 0 && bi < st.nten(), SADMRG_ERR_ARG, "tensor desc: block index out of range");
    SADMRG_REQUIRE(i == 0 || bi > t->block_index[i - 1], SADMRG_ERR_ARG, "tensor desc: block indices must ascend");
    int q[8], d[8];
    SADMRG_REQUIRE(st.block(bi, q, d), SADMRG_ERR_ARG, "tensor desc: block not allowed by symmetry");
    pres[bi] = 1;
  }
  BTensor<S> r = ops::from_host<S>(c, st, pres, static_cast<const S*>(t->data));
  // small operators keep a host copy (site operators are read on the host)
  if (r.nelem <= 64 && t->data) r.host.assign(static_cast<const S*>(t->data), static_cast<const S*>(t->data) + r.nelem);
  return r;
}

template <class S>
static State<S>& st_of(sadmrg_handle* h);
template <> State<double>& st_of<double>(sadmrg_handle* h) { return h->sd; }
template <> State<dcmplex>& st_of<dcmplex>(sadmrg_handle* h) { return h->sz; }

// After a bounded wait ran out, the persistent plans' split-K and dependency
// counters are part-way: zero them so the next call computes normally.
static void reset_plan_counters(sadmrg_handle* h) {
  auto reset = [&](auto& S_) {
    if (S_.heff) S_.heff->plan.reset_counters(h->ctx);
    if (S_.batch) S_.batch->merged.plan.reset_counters(h->ctx);
  };
  reset(h->sd);
  reset(h->sz);
  SADMRG_CUDA(cudaStreamSynchronize(h->ctx.stream));
}

// A tcgen05 item kernel whose bounded wait ran out leaves its tile unwritten and
// raises a device status word; calls that synchronise anyway check it.
static void check_device_status(sadmrg_handle* h) {
  const int v = umma_status(true);
  if (v < 0) throw Error(SADMRG_ERR_CUDA, "cannot read the tcgen05 status word");
  if (v != 0) {
    reset_plan_counters(h);
    throw Error(SADMRG_ERR_CUDA, "tcgen05 GEMM: a bounded wait ran out (status " + std::to_string(v) +
                                     "); the results of this call are invalid");
  }
}

template <class F>
static int dispatch(sadmrg_handle* h, F&& f) {
  return guard(h, [&]() {
    if (h->ctx.cplx) f((dcmplex*)nullptr);
    else f((double*)nullptr);
  });
}

extern "C" {

int sadmrg_version(void) { return 10000; }

int sadmrg_device_status(sadmrg_handle* h, int* status) {
  return guard(h, [&]() {
    SADMRG_REQUIRE(status, SADMRG_ERR_ARG, "device_status: null output");
    SADMRG_CUDA(cudaStreamSynchronize(h->ctx.stream));
    const int v = umma_status(true);
    SADMRG_REQUIRE(v >= 0, SADMRG_ERR_CUDA, "device_status: cannot read the status word");
    if (v != 0) reset_plan_counters(h);
    *status = v;
  });
}

int sadmrg_heff_wait_fault_test(sadmrg_handle* h, long long wait_ns, int* status) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "wait_fault_test: no plan");
    SADMRG_REQUIRE(status && wait_ns >= 1000000 && wait_ns <= 2000000000LL, SADMRG_ERR_ARG,
                   "wait_fault_test: wait_ns outside [1 ms, 2 s]");
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    SADMRG_REQUIRE(umma_status(true) == 0, SADMRG_ERR_STATE, "wait_fault_test: status word already set");
    const HeffPlan<S>& H = *S_.heff;
    Bases b{};
    b.p[0] = S_.io.get();
    b.p[1] = S_.io.template as<S>() + H.n;
    b.p[2] = H.opsbuf->get();
    b.p[3] = H.scratch->get();
    SADMRG_CUDA(cudaMemsetAsync(S_.io.get(), 0, sizeof(S) * H.n, c.stream));
    H.plan.run_starved(c, ScalarInfo<S>::cplx, b, 0, wait_ns);
    const int v = umma_status(true);
    SADMRG_REQUIRE(v >= 0, SADMRG_ERR_CUDA, "wait_fault_test: cannot read the status word");
    reset_plan_counters(h);
    *status = v;
  });
}

int sadmrg_create(int sym, int cplx, int device, sadmrg_handle** out) {
  if (!out || (sym != 0 && sym != 1)) return SADMRG_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return SADMRG_ERR_CUDA;
  if (device < 0 || device >= ndev) return SADMRG_ERR_ARG;
  auto* h = new (std::nothrow) sadmrg_handle();
  if (!h) return SADMRG_ERR_NOMEM;
  h->device = device;
  h->ctx.sym = sym ? Sym::SU2 : Sym::U1;
  h->ctx.cplx = cplx != 0;
  const int rc = guard(h, [&]() {
    SADMRG_CUDA(cudaStreamCreateWithFlags(&h->ctx.stream, cudaStreamNonBlocking));
    // Plans, Krylov spaces and SVD work buffers are allocated and freed once per
    // bond (stream-ordered).  With the pool's default release threshold (0) every
    // synchronisation hands the freed memory back to the driver and the next bond
    // maps it again, which costs milliseconds per bond; keep it cached in this
    // process instead (sadmrg_destroy trims the pool).
    {
      cudaMemPool_t pool;
      SADMRG_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
      uint64_t keep = UINT64_MAX;
      SADMRG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    SADMRG_CUDA(cudaMalloc(&h->ctx.d_scalars, 64 * sizeof(double)));
    SADMRG_CUDA(cudaMalloc(&h->ctx.d_partial, sizeof(double) * 2 * 512 * (size_t)h->ctx.npart));
    SADMRG_CUDA(cudaMalloc(&h->ctx.d_counter, sizeof(unsigned)));
    SADMRG_CUDA(cudaMemset(h->ctx.d_counter, 0, sizeof(unsigned)));
    SADMRG_CUDA(cudaMallocHost(&h->ctx.h_pinned, sizeof(double) * Ctx::kPinnedDoubles));
    if (h->ctx.sym == Sym::SU2) h->ctx.cgc = std::make_unique<CGCFactors>(1);
  });
  if (rc != SADMRG_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return SADMRG_OK;
}

int sadmrg_destroy(sadmrg_handle* h) {
  if (!h) return SADMRG_OK;
  cudaSetDevice(h->device);
  if (h->ctx.stream) cudaStreamSynchronize(h->ctx.stream);
  h->sd = State<double>();
  h->sz = State<dcmplex>();
  if (h->ctx.stream) {
    cudaStreamSynchronize(h->ctx.stream);
    cudaStreamDestroy(h->ctx.stream);
  }
  // hand the pool's cached, now unused memory back (memory of other live handles stays)
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, h->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
  delete h;
  return SADMRG_OK;
}

const char* sadmrg_last_error(const sadmrg_handle* h) { return h ? h->err.c_str() : "null handle"; }

int sadmrg_heff_plan(sadmrg_handle* h, const sadmrg_tensor_desc* psi, const sadmrg_tensor_desc* hhl,
                     const sadmrg_tensor_desc* hhr, int nops, const sadmrg_tensor_desc* opsd, int nterms,
                     const int* op1, const int* op2) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(psi && nops >= 0 && nterms >= 0 && (nops == 0 || opsd), SADMRG_ERR_ARG, "heff_plan: bad arguments");
    BTensor<S> p = from_desc<S>(c, psi);
    BTensor<S> hl, hr;
    if (hhl) hl = from_desc<S>(c, hhl);
    if (hhr) hr = from_desc<S>(c, hhr);
    std::vector<BTensor<S>> ov(nops);
    std::vector<const BTensor<S>*> opl(nops);
    for (int i = 0; i < nops; ++i) { ov[i] = from_desc<S>(c, &opsd[i]); opl[i] = &ov[i]; }
    std::vector<PairTerm> terms(nterms);
    for (int i = 0; i < nterms; ++i) {
      SADMRG_REQUIRE(op1[i] >= 0 && op1[i] < nops && op2[i] >= 0 && op2[i] < nops, SADMRG_ERR_ARG,
                     "heff_plan: operator index out of range");
      terms[i].op1 = op1[i];
      terms[i].op2 = op2[i];
    }
    auto& S_ = st_of<S>(h);
    S_.heff = std::make_unique<HeffPlan<S>>(build_heff<S>(c, p, hhl ? &hl : nullptr, hhr ? &hr : nullptr, opl, terms));
    S_.io.alloc(sizeof(S) * 2 * std::max<long long>(S_.heff->n, 1), c.stream);
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int sadmrg_set_lanczos_tol(sadmrg_handle* h, double ov_tol) {
  return guard(h, [&]() {
    SADMRG_REQUIRE(ov_tol > 0.0 && ov_tol < 1.0, SADMRG_ERR_ARG, "set_lanczos_tol: tolerance out of range");
    h->ctx.lanczos_ov_tol = ov_tol;
  });
}

int sadmrg_set_matvec_fusion(sadmrg_handle* h, int fused) {
  return guard(h, [&]() {
    SADMRG_REQUIRE(fused >= -1 && fused <= 1, SADMRG_ERR_ARG, "set_matvec_fusion: -1, 0 or 1");
    h->ctx.fused_matvec = fused;
  });
}

int sadmrg_heff_set_penalty(sadmrg_handle* h, int nvec, const void* vecs_host, const double* weights) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_set_penalty: no plan");
    SADMRG_REQUIRE(nvec >= 0 && nvec <= 512, SADMRG_ERR_ARG, "heff_set_penalty: 0 <= nvec <= 512");
    SADMRG_REQUIRE(nvec == 0 || (vecs_host && weights), SADMRG_ERR_ARG, "heff_set_penalty: null vectors or weights");
    HeffPlan<S>& H = *S_.heff;
    H.npen = 0;
    H.pen_o.reset();
    H.pen_wo.reset();
    H.pen_dot.reset();
    if (nvec == 0) return;
    const size_t bytes = sizeof(S) * (size_t)H.n * nvec;
    H.pen_o = std::make_shared<DevBuf>(bytes, c.stream);
    H.pen_wo = std::make_shared<DevBuf>(bytes, c.stream);
    H.pen_dot = std::make_shared<DevBuf>(sizeof(S) * (nvec + 1), c.stream);
    std::vector<S> wo((size_t)H.n * nvec);
    const S* o = static_cast<const S*>(vecs_host);
    for (int k = 0; k < nvec; ++k)
      for (long long i = 0; i < H.n; ++i) wo[(size_t)k * H.n + i] = o[(size_t)k * H.n + i] * weights[k];
    SADMRG_CUDA(cudaMemcpyAsync(H.pen_o->get(), vecs_host, bytes, cudaMemcpyHostToDevice, c.stream));
    SADMRG_CUDA(cudaMemcpyAsync(H.pen_wo->get(), wo.data(), bytes, cudaMemcpyHostToDevice, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    H.npen = nvec;
  });
}

int sadmrg_set_autotune(sadmrg_handle* h, int on) {
  return guard(h, [&]() { h->ctx.autotune = on ? 1 : 0; });
}

int sadmrg_set_svd_block(sadmrg_handle* h, int b) {
  return guard(h, [&]() {
    SADMRG_REQUIRE(b == 0 || b == 8 || b == 16, SADMRG_ERR_ARG, "set_svd_block: 0, 8 or 16");
    h->ctx.svd_block = b;
  });
}

int sadmrg_set_svd_stream(sadmrg_handle* h, int on) {
  return guard(h, [&]() { h->ctx.svd_stream = on ? 1 : 0; });
}

int sadmrg_set_svd_precondition(sadmrg_handle* h, int on) {
  return guard(h, [&]() {
    SADMRG_REQUIRE(on >= 0 && on <= 2, SADMRG_ERR_ARG, "set_svd_precondition: 0, 1 or 2");
    h->ctx.svd_qr = on;
  });
}

int sadmrg_set_tiles(sadmrg_handle* h, int bn, int kc_min, int kc_max, int ctas_per_sm, int one_launch) {
  return guard(h, [&]() {
    SADMRG_REQUIRE(bn == 0 || bn == 64 || bn == 128, SADMRG_ERR_ARG, "set_tiles: width must be 0, 64 or 128");
    SADMRG_REQUIRE(kc_min >= 0 && kc_max >= 0 && one_launch >= -1 && one_launch <= 1 &&
                       (ctas_per_sm == 1 || (ctas_per_sm == 2 && bn == 64)),
                   SADMRG_ERR_ARG, "set_tiles: arguments");
    UmmaTune t;
    t.bn = bn;
    t.kc_min = kc_min;
    t.kc_max = kc_max;
    t.ctas = ctas_per_sm;
    t.fused = one_launch;
    h->ctx.forced_tune = t;
  });
}

int sadmrg_heff_tiles(sadmrg_handle* h, int cap, double* out, int* n) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_tiles: no plan");
    SADMRG_REQUIRE(n && (cap <= 0 || out), SADMRG_ERR_ARG, "heff_tiles: null count or buffer");
    const GemmPlan& P = S_.heff->plan;
    const UmmaTune& t = P.tune;
    std::vector<double> v;
    const bool fused = P.runs_fused(h->ctx, ScalarInfo<S>::cplx, PREC_TF32X3);
    v.push_back(P.umma ? P.umma->bn : 0);
    v.push_back(t.kc_min);
    v.push_back(t.kc_max);
    v.push_back(P.umma ? P.umma->ctas : 1);
    v.push_back(fused ? 1 : 0);
    v.push_back(t.source);
    v.push_back(t.ncand);
    for (int i = 0; i < t.ncand; ++i) {
      v.push_back(t.cand_bn[i]);
      v.push_back(t.cand_kc[i]);
      v.push_back(t.cand_kmax[i]);
      v.push_back(t.cand_ctas[i]);
      v.push_back(t.cand_fused[i]);
      v.push_back(t.ms[i]);
    }
    *n = (int)v.size();
    for (int i = 0; i < cap && i < (int)v.size(); ++i) out[i] = v[i];
  });
}

int sadmrg_heff_info(sadmrg_handle* h, long long* n, double* flops, double* bytes, int* ntasks) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_info: no plan");
    if (n) *n = S_.heff->n;
    if (flops) *flops = (double)S_.heff->flops;
    if (bytes) *bytes = (double)S_.heff->bytes;
    if (ntasks) *ntasks = S_.heff->ntasks;
  });
}

int sadmrg_heff_apply(sadmrg_handle* h, const void* psi_host, void* out_host, int precision) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_apply: no plan");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "heff_apply: precision");
    const long long n = S_.heff->n;
    SADMRG_REQUIRE(n == 0 || (psi_host && out_host), SADMRG_ERR_ARG, "heff_apply: null buffer");
    S* din = S_.io.template as<S>();
    S* dout = din + n;
    SADMRG_CUDA(cudaMemcpyAsync(din, psi_host, sizeof(S) * n, cudaMemcpyHostToDevice, c.stream));
    S_.heff->apply(c, din, dout, precision);
    SADMRG_CUDA(cudaMemcpyAsync(out_host, dout, sizeof(S) * n, cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    check_device_status(h);
  });
}

int sadmrg_heff_apply_device(sadmrg_handle* h, const void* psi_dev, void* out_dev, int precision) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_apply_device: no plan");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "heff_apply: precision");
    SADMRG_REQUIRE(S_.heff->n == 0 || (psi_dev && out_dev), SADMRG_ERR_ARG, "heff_apply_device: null buffer");
    S_.heff->apply(h->ctx, static_cast<const S*>(psi_dev), static_cast<S*>(out_dev), precision);
  });
}

// Same matvec as sadmrg_heff_apply_device, but the products of stage 0 and the
// split-K partial tiles go to the library's fixed device scratch instead of the
// plan's buffers, so this call allocates nothing (see include/sadmrg.h).
int sadmrg_heff_apply_noalloc(sadmrg_handle* h, const void* psi_dev, void* out_dev, int precision) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_apply_noalloc: no plan");
    SADMRG_REQUIRE(psi_dev && out_dev, SADMRG_ERR_ARG, "heff_apply_noalloc: null device pointer");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG,
                   "heff_apply_noalloc: precision");
    const HeffPlan<S>& H = *S_.heff;
    const size_t xbytes = ((size_t)H.plan.scratch_elems * sizeof(S) + 255) & ~size_t(255);
    const size_t need = xbytes + H.plan.work_bytes(ScalarInfo<S>::cplx, precision);
    if (need > kNoAllocScratchBytes)
      throw Error(SADMRG_ERR_LIMIT, "heff_apply_noalloc: the plan needs " + std::to_string(need) +
                                        " bytes of scratch, more than the fixed " +
                                        std::to_string(kNoAllocScratchBytes) + " bytes");
    void* scratch = nullptr;
    const int rc = noalloc_scratch(&scratch);
    if (rc != 0)
      throw Error(SADMRG_ERR_CUDA, std::string("heff_apply_noalloc: cudaGetSymbolAddress: ") +
                                       cudaGetErrorString((cudaError_t)rc));
    Bases b{};
    b.p[0] = const_cast<void*>(psi_dev);
    b.p[1] = out_dev;
    b.p[2] = H.opsbuf->get();
    b.p[3] = scratch;
    H.plan.run(h->ctx, ScalarInfo<S>::cplx, precision, b, 0, -1, static_cast<unsigned char*>(scratch) + xbytes);
    H.penalty(h->ctx, static_cast<const S*>(psi_dev), static_cast<S*>(out_dev));
  });
}

int sadmrg_heff_profile(sadmrg_handle* h, int precision, int reps, const void* psi_dev, void* out_dev, double* ms,
                        double* flops) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_profile: no plan");
    SADMRG_REQUIRE(reps >= 1 && ms && flops, SADMRG_ERR_ARG, "heff_profile: reps or null outputs");
    const HeffPlan<S>& H = *S_.heff;
    const S* in = psi_dev ? static_cast<const S*>(psi_dev) : S_.io.template as<S>();
    S* out = out_dev ? static_cast<S*>(out_dev) : S_.io.template as<S>() + H.n;
    Bases b{};
    b.p[0] = const_cast<S*>(in);
    b.p[1] = out;
    b.p[2] = H.opsbuf->get();
    b.p[3] = H.scratch->get();
    cudaEvent_t ev[3];
    for (auto& e : ev) SADMRG_CUDA(cudaEventCreate(&e));
    double acc[2] = {0.0, 0.0};
    for (int r = 0; r < reps; ++r) {
      SADMRG_CUDA(cudaEventRecord(ev[0], c.stream));
      H.plan.run(c, ScalarInfo<S>::cplx, precision, b, 0, 1);
      SADMRG_CUDA(cudaEventRecord(ev[1], c.stream));
      H.plan.run(c, ScalarInfo<S>::cplx, precision, b, 1, 2);
      SADMRG_CUDA(cudaEventRecord(ev[2], c.stream));
      SADMRG_CUDA(cudaEventSynchronize(ev[2]));
      float t0 = 0.f, t1 = 0.f;
      SADMRG_CUDA(cudaEventElapsedTime(&t0, ev[0], ev[1]));
      SADMRG_CUDA(cudaEventElapsedTime(&t1, ev[1], ev[2]));
      acc[0] += t0;
      acc[1] += t1;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    check_device_status(h);
    ms[0] = acc[0] / reps;
    ms[1] = acc[1] / reps;
    // algorithmic flops per stage
    double f[2] = {0.0, 0.0};
    const auto& P = H.plan;
    for (size_t j = 0; j < P.jobs.size(); ++j)
      for (auto& t : P.job_terms[j])
        f[P.job_stage[j]] += (ScalarInfo<S>::cplx ? 8.0 : 2.0) * P.jobs[j].m * (double)P.jobs[j].n * t.k;
    flops[0] = f[0];
    flops[1] = f[1];
  });
}

int sadmrg_heff_launch_profile(sadmrg_handle* h, int precision, int reps, const void* psi_dev, void* out_dev, int cap,
                               int* nlaunch, int* kind, double* ms) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_launch_profile: no plan");
    SADMRG_REQUIRE(reps >= 1 && nlaunch, SADMRG_ERR_ARG, "heff_launch_profile: arguments");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "heff_launch_profile: precision");
    const HeffPlan<S>& H = *S_.heff;
    const S* in = psi_dev ? static_cast<const S*>(psi_dev) : S_.io.template as<S>();
    S* out = out_dev ? static_cast<S*>(out_dev) : S_.io.template as<S>() + H.n;
    Bases b{};
    b.p[0] = const_cast<S*>(in);
    b.p[1] = out;
    b.p[2] = H.opsbuf->get();
    b.p[3] = H.scratch->get();
    std::vector<double> acc;
    std::vector<int> kinds;
    for (int r = 0; r < reps; ++r) {
      std::vector<std::pair<int, cudaEvent_t>> ev;
      cudaEvent_t start;
      SADMRG_CUDA(cudaEventCreate(&start));
      SADMRG_CUDA(cudaEventRecord(start, c.stream));
      c.prof = &ev;
      try {
        H.plan.run(c, ScalarInfo<S>::cplx, precision, b);
      } catch (...) {
        c.prof = nullptr;
        throw;
      }
      c.prof = nullptr;
      SADMRG_CUDA(cudaStreamSynchronize(c.stream));
      if (acc.empty()) {
        acc.assign(ev.size(), 0.0);
        for (auto& e : ev) kinds.push_back(e.first);
      }
      SADMRG_REQUIRE(acc.size() == ev.size(), SADMRG_ERR_STATE, "heff_launch_profile: launch count changed");
      cudaEvent_t prev = start;
      for (size_t i = 0; i < ev.size(); ++i) {
        float t = 0.f;
        SADMRG_CUDA(cudaEventElapsedTime(&t, prev, ev[i].second));
        acc[i] += t;
        prev = ev[i].second;
      }
      cudaEventDestroy(start);
      for (auto& e : ev) cudaEventDestroy(e.second);
    }
    check_device_status(h);
    *nlaunch = (int)acc.size();
    for (int i = 0; i < (int)acc.size() && i < cap; ++i) {
      if (kind) kind[i] = kinds[i];
      if (ms) ms[i] = acc[i] / reps;
    }
  });
}

int sadmrg_heff_graph_steps(sadmrg_handle* h, int precision, int steps, const void* psi_dev, void* out_dev,
                            void* flush_dev, long long flush_bytes, double* ms) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_graph_steps: no plan");
    SADMRG_REQUIRE(steps >= 1 && ms && flush_bytes >= 0 && (flush_dev || flush_bytes == 0), SADMRG_ERR_ARG,
                   "heff_graph_steps: arguments");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "heff_graph_steps: precision");
    const HeffPlan<S>& H = *S_.heff;
    Bases b{};
    b.p[0] = const_cast<void*>(psi_dev ? psi_dev : S_.io.get());
    b.p[1] = out_dev ? out_dev : static_cast<void*>(S_.io.template as<S>() + H.n);
    b.p[2] = H.opsbuf->get();
    b.p[3] = H.scratch->get();
    // one plain run first: lazy one-time setup (kernel attributes, device queries) stays out of the capture
    H.plan.run(c, ScalarInfo<S>::cplx, precision, b);
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    SADMRG_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    try {
      H.plan.run(c, ScalarInfo<S>::cplx, precision, b);
    } catch (...) {
      cudaStreamEndCapture(c.stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    SADMRG_CUDA(cudaStreamEndCapture(c.stream, &g));
    const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(g);
      SADMRG_CUDA(ie);
    }
    std::vector<cudaEvent_t> ev(2 * (size_t)steps, nullptr);
    auto cleanup = [&]() {
      for (auto& e : ev)
        if (e) cudaEventDestroy(e);
      cudaGraphExecDestroy(ge);
      cudaGraphDestroy(g);
    };
    try {
      for (auto& e : ev) SADMRG_CUDA(cudaEventCreate(&e));
      const long long half = (flush_bytes / 2) & ~15LL;
      for (int r = 0; r < steps; ++r) {
        // evict the operands from L2 before the step, outside the events: write the
        // first half of the flush buffer, then read the second half, so that the
        // written lines are back in memory before the step starts
        if (half > 0) {
          SADMRG_CUDA(cudaMemsetAsync(flush_dev, r & 0xff, (size_t)half, c.stream));
          launch_read(static_cast<unsigned char*>(flush_dev) + half, half, h->ctx.d_counter, c.stream);
        }
        SADMRG_CUDA(cudaEventRecord(ev[2 * r], c.stream));
        SADMRG_CUDA(cudaGraphLaunch(ge, c.stream));
        SADMRG_CUDA(cudaEventRecord(ev[2 * r + 1], c.stream));
      }
      SADMRG_CUDA(cudaEventSynchronize(ev[2 * steps - 1]));
      for (int r = 0; r < steps; ++r) {
        float t = 0.f;
        SADMRG_CUDA(cudaEventElapsedTime(&t, ev[2 * r], ev[2 * r + 1]));
        ms[r] = t;
      }
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
    c.launches += (long long)H.plan.launches_per_run(ScalarInfo<S>::cplx, precision,
                                                   H.plan.runs_fused(c, ScalarInfo<S>::cplx, precision)) * (steps + 1);
    check_device_status(h);
  });
}

int sadmrg_heff_launches_per_matvec(sadmrg_handle* h, int precision, int* n) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.heff && n, SADMRG_ERR_ARG, "heff_launches_per_matvec: no plan");
    const HeffPlan<S>& H = *S_.heff;
    *n = H.plan.launches_per_run(ScalarInfo<S>::cplx, precision,
                                 H.plan.runs_fused(h->ctx, ScalarInfo<S>::cplx, precision)) +
         (H.npen > 0 ? 3 : 0);
  });
}

int sadmrg_heff_graph_bench(sadmrg_handle* h, int precision, int reps, const void* psi_dev, void* out_dev,
                            double* ms) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_graph_bench: no plan");
    SADMRG_REQUIRE(reps >= 1 && ms, SADMRG_ERR_ARG, "heff_graph_bench: arguments");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "heff_graph_bench: precision");
    const HeffPlan<S>& H = *S_.heff;
    Bases b{};
    b.p[0] = const_cast<void*>(psi_dev ? psi_dev : S_.io.get());
    b.p[1] = out_dev ? out_dev : static_cast<void*>(S_.io.template as<S>() + H.n);
    b.p[2] = H.opsbuf->get();
    b.p[3] = H.scratch->get();
    // one plain run first: lazy one-time setup (kernel attributes, device queries) stays out of the capture
    H.plan.run(c, ScalarInfo<S>::cplx, precision, b);
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    SADMRG_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
    try {
      H.plan.run(c, ScalarInfo<S>::cplx, precision, b);
    } catch (...) {
      cudaStreamEndCapture(c.stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    SADMRG_CUDA(cudaStreamEndCapture(c.stream, &g));
    const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(g);
      SADMRG_CUDA(ie);
    }
    cudaEvent_t e0, e1;
    SADMRG_CUDA(cudaEventCreate(&e0));
    SADMRG_CUDA(cudaEventCreate(&e1));
    SADMRG_CUDA(cudaGraphLaunch(ge, c.stream));   // warm
    SADMRG_CUDA(cudaEventRecord(e0, c.stream));
    for (int r = 0; r < reps; ++r) SADMRG_CUDA(cudaGraphLaunch(ge, c.stream));
    SADMRG_CUDA(cudaEventRecord(e1, c.stream));
    SADMRG_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    SADMRG_CUDA(cudaEventElapsedTime(&t, e0, e1));
    *ms = t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    c.launches += (long long)H.plan.launches_per_run(ScalarInfo<S>::cplx, precision,
                                                   H.plan.runs_fused(c, ScalarInfo<S>::cplx, precision)) * (reps + 1);
    check_device_status(h);
  });
}

int sadmrg_heff_lanczos(sadmrg_handle* h, void* psi_host, int mlanc, int precision, double* energy, int* matvecs) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_lanczos: no plan");
    SADMRG_REQUIRE(mlanc >= 2, SADMRG_ERR_ARG, "heff_lanczos: mlanc < 2");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "heff_lanczos: precision");
    const long long n = S_.heff->n;
    SADMRG_REQUIRE(n == 0 || psi_host, SADMRG_ERR_ARG, "heff_lanczos: null vector");
    S* dv = S_.io.template as<S>();
    SADMRG_CUDA(cudaMemcpyAsync(dv, psi_host, sizeof(S) * n, cudaMemcpyHostToDevice, c.stream));
    LanczosStats st = lanczos_solve<S>(c, *S_.heff, dv, mlanc, precision);
    SADMRG_CUDA(cudaMemcpyAsync(psi_host, dv, sizeof(S) * n, cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    check_device_status(h);
    if (energy) *energy = st.energy;
    if (matvecs) *matvecs = st.matvecs;
  });
}

int sadmrg_heff_lanczos2(sadmrg_handle* h, void* psi_host, int mlanc, double* energy, int* matvecs) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.heff, SADMRG_ERR_STATE, "heff_lanczos2: no plan");
    SADMRG_REQUIRE(mlanc >= 2, SADMRG_ERR_ARG, "heff_lanczos2: mlanc < 2");
    const long long n = S_.heff->n;
    SADMRG_REQUIRE(n == 0 || psi_host, SADMRG_ERR_ARG, "heff_lanczos2: null vector");
    S* dv = S_.io.template as<S>();
    SADMRG_CUDA(cudaMemcpyAsync(dv, psi_host, sizeof(S) * n, cudaMemcpyHostToDevice, c.stream));
    LanczosStats st = lanczos2<S>(c, *S_.heff, dv, mlanc);
    SADMRG_CUDA(cudaMemcpyAsync(psi_host, dv, sizeof(S) * n, cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    check_device_status(h);
    if (energy) *energy = st.energy;
    if (matvecs) *matvecs = st.matvecs;
  });
}

// ---- many instances in one launch ------------------------------------------
int sadmrg_batch_add(sadmrg_handle* h, sadmrg_handle* inst) {
  if (!inst) return h ? fail(h, SADMRG_ERR_ARG, "batch_add: null instance") : SADMRG_ERR_ARG;
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    SADMRG_REQUIRE(inst->device == h->device && inst->ctx.sym == h->ctx.sym && inst->ctx.cplx == h->ctx.cplx,
                   SADMRG_ERR_ARG, "batch_add: instance on another device or of another symmetry / scalar type");
    auto& I = st_of<S>(inst);
    SADMRG_REQUIRE(I.heff, SADMRG_ERR_STATE, "batch_add: the instance has no H_eff plan");
    auto& S_ = st_of<S>(h);
    if (!S_.batch) S_.batch = std::make_unique<HeffBatch<S>>();
    S_.batch->add(h->ctx, *I.heff);
  });
}

int sadmrg_batch_finalize(sadmrg_handle* h) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.batch, SADMRG_ERR_STATE, "batch_finalize: no instances added");
    S_.batch->finalize(h->ctx);
  });
}

int sadmrg_batch_clear(sadmrg_handle* h) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    st_of<S>(h).batch.reset();
  });
}

int sadmrg_batch_info(sadmrg_handle* h, int* ninst, long long* n, double* flops, int cap, long long* offsets) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.batch && S_.batch->ready, SADMRG_ERR_STATE, "batch_info: not finalized");
    const HeffBatch<S>& B = *S_.batch;
    if (ninst) *ninst = B.nseg();
    if (n) *n = B.merged.n;
    if (flops) *flops = (double)B.merged.flops;
    if (offsets)
      for (int i = 0; i < cap && i < (int)B.seg.size(); ++i) offsets[i] = B.seg[i];
  });
}

int sadmrg_batch_apply(sadmrg_handle* h, const void* psi_host, void* out_host, int precision) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.batch && S_.batch->ready, SADMRG_ERR_STATE, "batch_apply: not finalized");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "batch_apply: precision");
    const HeffPlan<S>& H = S_.batch->merged;
    SADMRG_REQUIRE(H.n == 0 || (psi_host && out_host), SADMRG_ERR_ARG, "batch_apply: null buffer");
    DevBuf io(sizeof(S) * 2 * std::max<long long>(H.n, 1), c.stream);
    S* din = io.as<S>();
    S* dout = din + H.n;
    SADMRG_CUDA(cudaMemcpyAsync(din, psi_host, sizeof(S) * H.n, cudaMemcpyHostToDevice, c.stream));
    H.apply(c, din, dout, precision);
    SADMRG_CUDA(cudaMemcpyAsync(out_host, dout, sizeof(S) * H.n, cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    check_device_status(h);
  });
}

int sadmrg_batch_profile(sadmrg_handle* h, int precision, int reps, double* ms) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.batch && S_.batch->ready, SADMRG_ERR_STATE, "batch_profile: not finalized");
    SADMRG_REQUIRE(reps >= 1 && ms, SADMRG_ERR_ARG, "batch_profile: arguments");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "batch_profile: precision");
    const HeffPlan<S>& H = S_.batch->merged;
    DevBuf io(sizeof(S) * 2 * std::max<long long>(H.n, 1), c.stream);
    SADMRG_CUDA(cudaMemsetAsync(io.get(), 0, sizeof(S) * 2 * std::max<long long>(H.n, 1), c.stream));
    S* din = io.as<S>();
    H.apply(c, din, din + H.n, precision);   // warm
    cudaEvent_t e0, e1;
    SADMRG_CUDA(cudaEventCreate(&e0));
    SADMRG_CUDA(cudaEventCreate(&e1));
    SADMRG_CUDA(cudaEventRecord(e0, c.stream));
    for (int r = 0; r < reps; ++r) H.apply(c, din, din + H.n, precision);
    SADMRG_CUDA(cudaEventRecord(e1, c.stream));
    SADMRG_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    SADMRG_CUDA(cudaEventElapsedTime(&t, e0, e1));
    *ms = t / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_device_status(h);
  });
}

int sadmrg_batch_lanczos(sadmrg_handle* h, void* psi_host, int mlanc, int precision, double* energies, int* matvecs,
                         int* batched_matvecs) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(S_.batch && S_.batch->ready, SADMRG_ERR_STATE, "batch_lanczos: not finalized");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "batch_lanczos: precision");
    SADMRG_REQUIRE(mlanc >= 2, SADMRG_ERR_ARG, "batch_lanczos: mlanc < 2");
    const HeffBatch<S>& B = *S_.batch;
    SADMRG_REQUIRE(B.merged.n == 0 || psi_host, SADMRG_ERR_ARG, "batch_lanczos: null vector");
    DevBuf io(sizeof(S) * std::max<long long>(B.merged.n, 1), c.stream);
    SADMRG_CUDA(cudaMemcpyAsync(io.get(), psi_host, sizeof(S) * B.merged.n, cudaMemcpyHostToDevice, c.stream));
    BatchStats st = batch_lanczos_solve<S>(c, B, io.as<S>(), mlanc, precision);
    SADMRG_CUDA(cudaMemcpyAsync(psi_host, io.get(), sizeof(S) * B.merged.n, cudaMemcpyDeviceToHost, c.stream));
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
    check_device_status(h);
    for (int i = 0; i < B.nseg(); ++i) {
      if (energies) energies[i] = st.energy[i];
      if (matvecs) matvecs[i] = st.matvecs[i];
    }
    if (batched_matvecs) *batched_matvecs = st.launches_matvec;
  });
}

int sadmrg_svd_truncate(sadmrg_handle* h, const sadmrg_tensor_desc* psi, const sadmrg_tensor_desc* tu,
                        const sadmrg_tensor_desc* tv, double p1, double p2, int max_dcut, int* kept,
                        double* discarded_weight) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    Ctx& c = h->ctx;
    SADMRG_REQUIRE(max_dcut > 0, SADMRG_ERR_ARG, "svd_truncate: max_dcut must be positive");
    BTensor<S> p = from_desc<S>(c, psi), u = from_desc<S>(c, tu), v = from_desc<S>(c, tv);
    SvdStats s = block_svd<S>(c, p, u, p1, v, p2, max_dcut, nullptr);
    auto& S_ = st_of<S>(h);
    S_.staged[0] = std::move(u);
    S_.staged[1] = std::move(v);
    if (kept) *kept = s.kept;
    if (discarded_weight) *discarded_weight = s.discarded_weight;
  });
}

int sadmrg_chain_create(sadmrg_handle* h, int lx, int ly, int bondd, int physpn, int totspin, int open, double J2) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    SADMRG_REQUIRE(lx >= 1 && ly >= 1 && bondd >= 1, SADMRG_ERR_ARG, "chain_create: bad size");
    st_of<S>(h).chain = std::make_unique<Chain<S>>(h->ctx, lx, ly, bondd, physpn, totspin, open, J2);
  });
}

int sadmrg_chain_set_dm(sadmrg_handle* h, double dz) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    S_.chain->set_dm(dz);
  });
}

int sadmrg_chain_set_excited(sadmrg_handle* h, int exci) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    S_.chain->set_excited(exci);
  });
}

int sadmrg_chain_set_precision(sadmrg_handle* h, int precision) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    SADMRG_REQUIRE(precision == PREC_FP64 || precision == PREC_TF32X3, SADMRG_ERR_ARG, "precision");
    S_.chain->prec = precision;
  });
}

int sadmrg_chain_idmrg(sadmrg_handle* h, double* energy) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    S_.chain->do_idmrg();
    SADMRG_CUDA(cudaStreamSynchronize(h->ctx.stream));
    check_device_status(h);
    if (energy) *energy = S_.chain->energy();
  });
}

int sadmrg_chain_prepare_sweep(sadmrg_handle* h) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    S_.chain->prepare_sweep();
    SADMRG_CUDA(cudaStreamSynchronize(h->ctx.stream));
  });
}

int sadmrg_chain_sweep(sadmrg_handle* h, double* energy) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    S_.chain->sweep();
    SADMRG_CUDA(cudaStreamSynchronize(h->ctx.stream));
    check_device_status(h);
    if (energy) *energy = S_.chain->energy();
  });
}

int sadmrg_chain_read_mps(sadmrg_handle* h, const char* dir, int bond_read) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    SADMRG_REQUIRE(dir, SADMRG_ERR_ARG, "read_mps: null path");
    SADMRG_REQUIRE(S_.chain->read_mps(dir, bond_read), SADMRG_ERR_ARG, "read_mps: checkpoint files missing");
  });
}

int sadmrg_chain_save_mps(sadmrg_handle* h, const char* dir) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    SADMRG_REQUIRE(dir, SADMRG_ERR_ARG, "save_mps: null path");
    S_.chain->save_mps(dir);
  });
}

int sadmrg_chain_set_mlanc(sadmrg_handle* h, int mlanc) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    SADMRG_REQUIRE(mlanc >= 2 && mlanc <= 1000, SADMRG_ERR_ARG, "chain_set_mlanc: mlanc outside [2, 1000]");
    S_.chain->mlanc_max = mlanc;
  });
}

}  // extern "C"

// checkpoint files of the singular values and the energy: fn(chain, dir)
template <class F>
static int chain_file_op(sadmrg_handle* h, const char* dir, const char* what, F&& fn) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    SADMRG_REQUIRE(dir, SADMRG_ERR_ARG, std::string(what) + ": null path");
    fn(*S_.chain, std::string(dir));
  });
}

extern "C" {

int sadmrg_chain_save_ww(sadmrg_handle* h, const char* dir) {
  return chain_file_op(h, dir, "save_ww", [](auto& ch, const std::string& d) { ch.save_ww(d); });
}
int sadmrg_chain_read_ww(sadmrg_handle* h, const char* dir, int bond_read) {
  if (bond_read < 1) return fail(h, SADMRG_ERR_ARG, "read_ww: bond_read < 1");
  return chain_file_op(h, dir, "read_ww", [&](auto& ch, const std::string& d) { ch.read_ww(d, bond_read); });
}
int sadmrg_chain_save_enr(sadmrg_handle* h, const char* dir) {
  return chain_file_op(h, dir, "save_enr", [](auto& ch, const std::string& d) { ch.save_enr(d); });
}
int sadmrg_chain_read_enr(sadmrg_handle* h, const char* dir, int bond_read) {
  return chain_file_op(h, dir, "read_enr", [&](auto& ch, const std::string& d) { ch.read_enr(d, bond_read); });
}

int sadmrg_chain_ww(sadmrg_handle* h, int cap, int* n, double* out) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    SADMRG_REQUIRE(n && (cap <= 0 || out), SADMRG_ERR_ARG, "chain_ww: null count or buffer");
    const auto& w = S_.chain->ww;
    *n = (int)w.size();
    for (int i = 0; i < cap && i < (int)w.size(); ++i) out[i] = w[i];
  });
}

int sadmrg_chain_freeze(sadmrg_handle* h, int il, const char* export_dir) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    Ctx& c = h->ctx;
    BTensor<S> psi;
    S_.heff = std::make_unique<HeffPlan<S>>(S_.chain->freeze(il, psi));
    S_.io.alloc(sizeof(S) * 2 * std::max<long long>(S_.heff->n, 1), c.stream);
    S_.staged[0] = std::move(psi);
    if (export_dir && export_dir[0]) S_.chain->export_problem(il, S_.staged[0], export_dir);
    SADMRG_CUDA(cudaStreamSynchronize(c.stream));
  });
}

int sadmrg_chain_bond(sadmrg_handle* h, int site, int cap, int* nsec, int* q, int* d) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    SADMRG_REQUIRE(site >= 0 && site < S_.chain->ns, SADMRG_ERR_ARG, "chain_bond: site");
    SADMRG_REQUIRE(nsec && (cap <= 0 || (q && d)), SADMRG_ERR_ARG, "chain_bond: null count or buffers");
    const auto& u = S_.chain->uu[site];
    if (u.st.nbond() < 3) { *nsec = 0; return; }
    const Bond& b = u.st.bonds[2];
    *nsec = b.nmom();
    SADMRG_REQUIRE(b.nmom() <= cap, SADMRG_ERR_LIMIT, "chain_bond: capacity");
    for (int k = 0; k < b.nmom(); ++k) { q[k] = b.q[k]; d[k] = b.d[k]; }
  });
}

int sadmrg_chain_bond_flags(sadmrg_handle* h, int cap, int* flags) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain && flags, SADMRG_ERR_STATE, "chain_bond_flags: no chain");
    const auto& f = S_.chain->bond_flags;
    for (int i = 0; i < cap; ++i) flags[i] = i < (int)f.size() ? f[i] : 0;
  });
}

int sadmrg_chain_stats(sadmrg_handle* h, double* out, int n) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    SADMRG_REQUIRE(n <= 0 || out, SADMRG_ERR_ARG, "chain_stats: null buffer");
    const Timers& t = S_.chain->timers;
    const double v[14] = {t.lanczos, t.env, t.svd, t.prep, (double)t.matvecs, t.heff_flops,
                          (double)h->ctx.gemm_flops, (double)h->ctx.launches, S_.chain->last_discarded,
                          (double)S_.chain->near_ties, t.svd_kernel, (double)t.svd_sweeps, t.plan,
                          (double)S_.chain->stop_ties};
    for (int i = 0; i < n && i < 14; ++i) out[i] = v[i];
  });
}

int sadmrg_chain_set_tensor(sadmrg_handle* h, int kind, int site, int k, const sadmrg_tensor_desc* t) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    auto& ch = *S_.chain;
    SADMRG_REQUIRE(site >= 0 && site < ch.ns && k >= 0 && k < ch.ns, SADMRG_ERR_ARG, "set_tensor: index");
    BTensor<S> v = t ? from_desc<S>(h->ctx, t) : BTensor<S>();
    if (kind == 0) ch.uu[site] = std::move(v);
    else if (kind == 1) ch.hh[site] = std::move(v);
    else if (kind == 2) ch.opr[site][k] = std::move(v);
    else throw Error(SADMRG_ERR_ARG, "set_tensor: kind");
  });
}

int sadmrg_chain_stage_tensor(sadmrg_handle* h, int kind, int site, int k) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    auto& ch = *S_.chain;
    SADMRG_REQUIRE(site >= 0 && site < ch.ns && k >= 0 && k < ch.ns, SADMRG_ERR_ARG, "stage_tensor: index");
    const BTensor<S>* src = nullptr;
    if (kind == 0) src = &ch.uu[site];
    else if (kind == 1) src = &ch.hh[site];
    else if (kind == 2) src = &ch.opr[site][k];
    else throw Error(SADMRG_ERR_ARG, "stage_tensor: kind");
    S_.staged[0] = src->null() ? BTensor<S>() : clone(h->ctx, *src);
  });
}

int sadmrg_chain_env_update(sadmrg_handle* h, int site, int dir, int real_env) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    auto& S_ = st_of<S>(h);
    SADMRG_REQUIRE(S_.chain, SADMRG_ERR_STATE, "no chain");
    auto& ch = *S_.chain;
    SADMRG_REQUIRE(site >= 0 && site < ch.ns, SADMRG_ERR_ARG, "env_update: site");
    if (dir == 0) ch.prepare_site_operator_from_left(site, real_env != 0);
    else ch.prepare_site_operator_from_right(site, real_env != 0);
    SADMRG_CUDA(cudaStreamSynchronize(h->ctx.stream));
  });
}

int sadmrg_staged_info(sadmrg_handle* h, int which, int* nbond, int* locspin, int* nsectors, int* nblocks,
                       long long* nelem) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    SADMRG_REQUIRE(which == 0 || which == 1, SADMRG_ERR_ARG, "staged: which");
    SADMRG_REQUIRE(nbond && locspin && nsectors && nblocks && nelem, SADMRG_ERR_ARG, "staged_info: null output");
    const BTensor<S>& t = st_of<S>(h).staged[which];
    *nbond = t.st.nbond();
    *locspin = t.st.locspin;
    int ns = 0, nb = 0;
    for (auto& b : t.st.bonds) ns += b.nmom();
    for (long i = 0; i < t.nten(); ++i) nb += t.present(i) ? 1 : 0;
    *nsectors = ns;
    *nblocks = nb;
    *nelem = t.nelem;
  });
}

int sadmrg_staged_read(sadmrg_handle* h, int which, int* dir, int* nmom, int* q, int* d, long long* block_index,
                       void* data) {
  return dispatch(h, [&](auto* tag) {
    using S = std::remove_pointer_t<decltype(tag)>;
    SADMRG_REQUIRE(which == 0 || which == 1, SADMRG_ERR_ARG, "staged: which");
    const BTensor<S>& t = st_of<S>(h).staged[which];
    SADMRG_REQUIRE(t.st.nbond() == 0 || (dir && nmom && q && d), SADMRG_ERR_ARG, "staged_read: null bond buffers");
    long npresent = 0;
    for (long i = 0; i < t.nten(); ++i) npresent += t.present(i) ? 1 : 0;
    SADMRG_REQUIRE(npresent == 0 || block_index, SADMRG_ERR_ARG, "staged_read: null block_index");
    SADMRG_REQUIRE(t.nelem == 0 || data, SADMRG_ERR_ARG, "staged_read: null data");
    int o = 0;
    for (int b = 0; b < t.st.nbond(); ++b) {
      dir[b] = t.st.bonds[b].dir;
      nmom[b] = t.st.bonds[b].nmom();
      for (int k = 0; k < nmom[b]; ++k) { q[o] = t.st.bonds[b].q[k]; d[o] = t.st.bonds[b].d[k]; ++o; }
    }
    int nb = 0;
    for (long i = 0; i < t.nten(); ++i)
      if (t.present(i)) block_index[nb++] = i;
    if (t.nelem > 0)
      SADMRG_CUDA(cudaMemcpyAsync(data, t.data(), sizeof(S) * t.nelem, cudaMemcpyDeviceToHost, h->ctx.stream));
    SADMRG_CUDA(cudaStreamSynchronize(h->ctx.stream));
  });
}

}  // extern "C"
