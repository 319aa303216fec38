// tensor.hpp -- device-resident block-sparse tensors and the task-plan builder.
//
// A BTensor keeps the reference's block structure (Struct = bonds, directions,
// locspin; a block is present or null) on the host and all present blocks in
// one contiguous device buffer, in block-index order, each block column-major
// with bond 0 fastest (the reference's Dense layout, src/dense_inst.cpp:28-45).
// For SU(2) the blocks hold reduced matrix elements; the CGC blocks of the
// reference are never materialised, because every CGC the hot path needs is a
// standard one (make_cgc / identity / singlet) and its effect is a scalar
// factor folded into the task (src/block_tensor_inst.cpp:1433-1441, 2268-2272).
#pragma once
#include <cuda_runtime.h>
#include <memory>
#include <string>
#include <vector>

#include "cgc.hpp"
#include "common.hpp"
#include "kernels.cuh"
#include "symmetry.hpp"

namespace sadmrg {

// Tile choice of a plan's tcgen05 schedule.  Without tuning the heuristics
// decide (source 0); the autotuner (dmrg.cpp) times candidate schedules on the
// plan itself and keeps the fastest per block-size histogram (source 1 when it
// was timed for this plan, 2 when an earlier plan with the same histogram
// decided it, 3 when the caller set it).
struct UmmaTune {
  int bn = 0;          // output tile width 64 or 128; 0: 128 when the 128-wide tiles fill the GPU twice
  int kc_min = 16;     // fewest k slabs in a split-K chunk; 0: no split for balance (kc_max still applies)
  int kc_max = 0;      // most k slabs in one item (longer reductions are split); 0: no cap
  int fused = -1;      // 1: a whole matvec in one cooperative launch, 0: one launch per stage, -1: Ctx's setting
  int ctas = 1;        // CTAs per SM (2: width 64 only, a 2-stage ring each)
  int source = 0;
  int ncand = 0;       // candidates timed, with their device time (ms) per matvec
  float ms[8] = {};
  int cand_bn[8] = {}, cand_kc[8] = {}, cand_kmax[8] = {}, cand_fused[8] = {}, cand_ctas[8] = {};
};

struct Ctx {
  cudaStream_t stream = nullptr;
  Sym sym = Sym::U1;
  bool cplx = false;
  int physpn = 1;
  std::unique_ptr<CGCFactors> cgc;
  double* d_scalars = nullptr;   // small device scratch for reductions
  double* d_partial = nullptr;
  unsigned* d_counter = nullptr; // last-block counter of the one-launch reductions (zero between launches)
  double* h_pinned = nullptr;    // page-locked host scratch (kPinnedDoubles) for async scalar reads
  static constexpr int kPinnedDoubles = 4096;
  int npart = 296;
  double lanczos_ov_tol = 1e-8;  // stop when |<v|Hv>|/|Hv| is this close to 1 (src/dmrg_inst.cpp:1338)
  // tcgen05 matvec as one cooperative launch instead of pack + one launch per
  // stage: 1 always, 0 never, -1 (default) for plans below kAutoFuseFlops
  int fused_matvec = -1;
  static constexpr double kAutoFuseFlops = 4e9;
  // time tile candidates for every new H_eff plan (1) or use the heuristics (0)
  int autotune = 1;
  // block SVD: Householder QRs before the Jacobi: 0 never, 1 for calls whose widest
  // block has at least 32 columns, 2 always
  int svd_qr = 1;
  // block SVD: stream every Jacobi visit's rows in chunks (1) or keep the pair's
  // columns in shared memory where they fit (0)
  int svd_stream = 0;
  // block SVD: Jacobi column blocks of 8 or 16, or 0 for the rule in run_jacobi_svd
  int svd_block = 0;
  // a tile choice every new H_eff plan takes instead (bn > 0), e.g. to profile one
  UmmaTune forced_tune;
  const int* job_mask = nullptr; // device flags per job tag; GemmPlan::run skips jobs whose flag is 0
  long long gemm_flops = 0;      // running counter of algorithmic GEMM flops issued
  long long launches = 0;        // kernels launched by this context
  // when set, GemmPlan::run records an event after every launch (what ran, event)
  std::vector<std::pair<int, cudaEvent_t>>* prof = nullptr;
  ~Ctx();
};

template <class S>
struct BTensor {
  Struct st;
  std::vector<long long> off;  // element offset of each block, -1 if null
  long long nelem = 0;
  std::shared_ptr<DevBuf> buf;
  std::vector<S> host;         // host mirror, only kept for tiny local operators

  bool null() const { return st.nbond() == 0; }
  S* data() const { return buf ? buf->as<S>() : nullptr; }
  bool present(long b) const { return b >= 0 && b < (long)off.size() && off[b] >= 0; }
  long nten() const { return (long)off.size(); }
};

struct Blk {
  long idx;
  int q[4];
  int d[4];
  long long off;
  long long rows() const { return (long long)d[0] * (d[1] > 0 ? d[1] : 1); }  // for 3-leg (d0*d1) x d2
};

// allowed and present blocks in block-index order
template <class S> std::vector<Blk> blocks_of(const BTensor<S>& t);

// allocate a tensor whose present blocks are flagged; zero-filled
template <class S> BTensor<S> alloc_tensor(Ctx& c, const Struct& st, const std::vector<char>& present);
template <class S> BTensor<S> clone(Ctx& c, const BTensor<S>& t);

// Work items and split-K reductions of a plan for the mma.sync item kernels.
struct GemmSchedule {
  int bm = 64, bn = 64;
  std::vector<WorkItem> items;
  std::vector<RedItem> reds;
  std::vector<int> stage_items;   // item offsets per stage (size nstage+1)
  std::vector<int> stage_reds;    // reduction offsets per stage (size nstage+1)
  WorkItem* d_items = nullptr;
  RedItem* d_reds = nullptr;
  std::shared_ptr<DevBuf> work;   // split-K partial tiles
  std::shared_ptr<DevBuf> tile_cnt;   // per RedItem: items finished in the current launch
  int nslot = 0;
  size_t work_bytes() const { return work ? work->bytes() : 0; }
};

// The tcgen05 schedule of a plan: operand panels, panel-addressed terms, jobs,
// slab-granular items (umma.cu); complex plans run in the real form of every
// product (kernels.cuh).  Built only when every term fits the panel scheme
// (constant operands in buffer 2, psi in buffer 0, stage-0 results in buffer 3
// consumed only as untransposed A operands with one real alpha each, other
// terms with coefficient 1).
struct UmmaSchedule {
  int bn = 64;
  int ctas = 1;                            // CTAs per SM of its launches
  std::vector<PackJob> cpack, vpack;       // constant panels (packed once), psi panels (every apply)
  long long cchunks = 0, vchunks = 0;      // multiples of 256 (one block per 256 chunks)
  std::vector<int> cblk, vblk;             // block -> pack job
  std::vector<UTerm> terms;
  std::vector<UJob> jobs;
  std::vector<UItem> items;
  std::vector<URed> reds;
  std::vector<int> stage_items, stage_reds;
  std::shared_ptr<DevBuf> dev, pconst, pvar, slots, tile_cnt, deps;
  std::vector<int> dep_target;             // per dependency counter: its value when the panels are complete
  int* d_dep_target = nullptr;
  PackJob* d_vpack = nullptr;
  int* d_vblk = nullptr;
  UTerm* d_terms = nullptr;
  UJob* d_jobs = nullptr;
  UItem* d_items = nullptr;
  URed* d_reds = nullptr;
  int nslot = 0;
  size_t slot_bytes() const { return slots ? slots->bytes() : 0; }
};

// A task plan: stage-0 jobs write scratch products, stage-1 jobs the outputs.
struct GemmPlan {
  std::vector<std::vector<GemmTerm>> job_terms;
  std::vector<GemmJob> jobs;
  std::vector<int> job_stage;
  long long scratch_elems = 0;
  int nstage = 2;
  // device copy
  std::vector<GemmTerm> flat_terms;
  GemmSchedule sched;                  // mma.sync items (FP64, and 3xTF32 when there is no tcgen05 schedule)
  std::shared_ptr<UmmaSchedule> umma;  // tcgen05 3xTF32 (real plans finalised with mixed = true)
  std::shared_ptr<DevBuf> dev;
  GemmTerm* d_terms = nullptr;
  GemmJob* d_jobs = nullptr;
  long long flops = 0;            // algorithmic flops of one execution (real multiply-adds * 2)
  int target_items = 148 * 8;     // work items per stage the split-K aims for
  UmmaTune tune;                  // tcgen05 tile choice (build_umma reads it)
  Bases const_bases{};            // where the constant panels come from (kept for rebuilds)

  int add_job(int stage, int cbuf, long long coff, int m, int n, int ldc, int flags);
  void add_term(int job, int abuf, long long aoff, int lda, int bbuf, long long boff, int ldb, int k, int flags,
                double ar, double ai);
  long long alloc_scratch(long long elems) { long long o = scratch_elems; scratch_elems += elems; return o; }
  // mixed: also build the tcgen05 schedule; its constant panels are packed from
  // const_bases (buffer 2) on the context's stream.
  void finalize(Ctx& c, bool cplx, bool mixed = false, const Bases* const_bases = nullptr);
  bool uses_umma(bool /*cplx*/, int prec) const { return prec == PREC_TF32X3 && umma != nullptr; }
  void run(Ctx& c, bool cplx, int prec, const Bases& b, int stage_lo = 0, int stage_hi = -1,
           void* work_override = nullptr) const;
  // bytes of split-K workspace a run at this precision uses
  size_t work_bytes(bool cplx, int prec) const {
    return uses_umma(cplx, prec) ? umma->slot_bytes() : sched.work_bytes();
  }
  int launches_per_run(bool cplx, int prec, bool fused) const;
  // Zero the split-K tile counters and the tcgen05 dependency counters.  A launch
  // whose bounded wait ran out leaves them part-way (its aborted items never
  // count in), and the next run would emit tiles too early.
  void reset_counters(Ctx& c) const;
  // Failure-path check of the bounded waits: the whole split-precision matvec as
  // one cooperative launch in which dependency counter `starve` can never reach
  // its target (the target is raised by one for this launch), every wait limited
  // to wait_ns.  Leaves the status word set; the caller resets the counters.
  void run_starved(Ctx& c, bool cplx, const Bases& b, int starve, long long wait_ns) const;
  // whether run() takes the single-launch path for a whole matvec under c's setting
  bool runs_fused(const Ctx& c, bool cplx, int prec) const;
  bool empty() const { return jobs.empty(); }
  // the tcgen05 schedule again with the current `tune` (false: the plan has none)
  bool rebuild_umma(Ctx& c, bool cplx);
  // block-size histogram of the plan -- jobs bucketed by stage and log2 of m, n
  // and their total k, bucket counts by log2: the key of the tile-choice cache
  std::string tune_key(bool cplx) const;

 private:
  void build_schedule(GemmSchedule& s, bool cplx);
  bool build_umma(Ctx& c, const Bases& cb, bool cplx);
};

}  // namespace sadmrg
