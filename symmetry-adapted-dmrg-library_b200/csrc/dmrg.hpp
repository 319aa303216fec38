// dmrg.hpp -- two-site DMRG driver on device-resident block tensors.
//
// Mirrors the reference's DMRG<Scalar,Sym> / Lanczos<Scalar,Sym> control flow
// (dmrg.hpp, src/dmrg_inst.cpp) step for step: iDMRG warm-up, prepare_sweep,
// sweep (left, right, return passes), with every data-bearing operation run on
// the GPU and only sector bookkeeping on the host.
#pragma once
#include <array>
#include <map>
#include <chrono>
#include <random>
#include <string>

#include "ops.hpp"

namespace sadmrg {

// H_eff * psi for a fixed two-site problem: all sector products of one matvec
// in two grouped launches (stage 0: X = op1^T psi; stage 1: out = sum f X op2
// + diagonal terms), built once per bond and replayed for every Lanczos step.
template <class S>
struct HeffPlan {
  GemmPlan plan;
  std::shared_ptr<DevBuf> opsbuf;    // packed operator data
  std::shared_ptr<DevBuf> scratch;
  Struct psi_st;
  std::vector<long long> psi_off;
  long long n = 0;                   // psi elements
  long long flops = 0;               // algorithmic flops per matvec
  long long bytes = 0;               // psi in + out + operators, once
  int ntasks = 0;
  // excited-state penalty (src/dmrg_inst.cpp:352-363): out -= sum_k w_k <o_k|psi> o_k,
  // o_k the lower states in this two-site basis, w_k their energies
  int npen = 0;
  std::shared_ptr<DevBuf> pen_o;     // npen vectors o_k, psi layout
  std::shared_ptr<DevBuf> pen_wo;    // w_k o_k
  std::shared_ptr<DevBuf> pen_dot;   // <o_k|psi>
  void apply(Ctx& c, const S* psi, S* out, int prec) const;
  void penalty(Ctx& c, const S* psi, S* out) const;
};

struct PairTerm {
  int op1 = -1, op2 = -1;            // indices into the operator list
};

template <class S>
// tune: time the tcgen05 schedule candidates for this plan (autotuner, dmrg.cpp) when
// the context allows it -- worth it for a plan applied many times, not for the
// ~25 matvecs of one sweep step
HeffPlan<S> build_heff(Ctx& c, const BTensor<S>& psi, const BTensor<S>* hhL, const BTensor<S>* hhR,
                       const std::vector<const BTensor<S>*>& opl, const std::vector<PairTerm>& terms,
                       bool tune = true);

struct LanczosStats {
  int matvecs = 0;
  int matvecs_fp64 = 0;
  int iters = 0;
  double energy = 0.0;
  double overlap = 0.0;
};

// Lanczos::lanczos1 (src/dmrg_inst.cpp:1286-1348) on device vectors.
// v (length n) holds the start vector on entry and the Ritz vector on exit.
// residual_test: at the check points stop on the Lanczos residual estimate
// b_m |z_m| instead of the reference's check matvec, with check points every
// check_every steps (the reference: 4); used by the mixed solver only.
template <class S>
LanczosStats lanczos1(Ctx& c, const HeffPlan<S>& H, S* v, int mlanc, int prec, bool residual_test = false,
                      int check_every = 4, bool variant2 = false);
// Lanczos::lanczos2 (src/dmrg_inst.cpp:1352-1397), FP64: the same recurrence with
// full reorthogonalisation but no convergence checks -- all mlanc steps, the
// energy and Ritz vector of the full tridiagonal; a breakdown (b < 1e-6, from
// step 2) returns the Ritz pair of the steps before it.
template <class S>
LanczosStats lanczos2(Ctx& c, const HeffPlan<S>& H, S* v, int mlanc);
// Mixed precision: lanczos1 with 3xTF32 matvecs, then an FP64 restart from
// its Ritz vector (defect correction) so the energy is an FP64 Lanczos result.
template <class S>
LanczosStats lanczos_solve(Ctx& c, const HeffPlan<S>& H, S* v, int mlanc, int prec);

// symmetric tridiagonal eigenproblem: d diagonal (ascending on return), e[i]
// coupling of i and i+1, z column-major eigenvectors (dmrg.cpp)
void tridiag_eig(int n, std::vector<double>& d, std::vector<double> e, std::vector<double>& z);

// Many independent frozen two-site problems merged into one plan: their vectors
// lie back to back (segment s = [seg[s], seg[s+1])) and one launch per stage
// runs the sector products of all of them (batch.cpp).
template <class S>
struct HeffBatch {
  struct Part {
    std::vector<std::vector<GemmTerm>> job_terms;
    std::vector<GemmJob> jobs;
    std::vector<int> job_stage;
    long long scratch = 0, n = 0, flops = 0;
    std::shared_ptr<DevBuf> ops;     // the instance's packed operators (kept alive until finalize)
  };
  std::vector<Part> parts;
  HeffPlan<S> merged;
  std::vector<long long> seg;        // nseg + 1 offsets
  std::shared_ptr<DevBuf> d_seg;
  bool ready = false;
  void add(Ctx& c, const HeffPlan<S>& H);
  void finalize(Ctx& c);
  int nseg() const { return (int)seg.size() - 1; }
};

struct BatchStats {
  std::vector<double> energy;        // per instance
  std::vector<int> matvecs;          // per instance (matvecs taken while it was not converged)
  int launches_matvec = 0;           // batched matvecs (each one launch per stage for all instances)
};

// Lanczos::lanczos1 on every instance at once: the same recurrence and checks as
// lanczos1 per segment; instances that converge keep their Ritz vector in v.
// prec TF32X3: split-precision phase then an FP64 restart, as lanczos_solve.
template <class S>
BatchStats batch_lanczos_solve(Ctx& c, const HeffBatch<S>& B, S* v, int mlanc, int prec);

struct SvdStats {
  int kept = 0;
  double discarded_weight = 0.0;
  int sweeps_max = 0;
  double jacobi_s = 0.0;       // wall time of the Jacobi solve
  double jacobi_kernel_ms = -1.0;
  int max_rows = 0, max_cols = 0;
  bool near_tie = false;      // the D-th and (D+1)-th singular values agree to 1e-8 (relative), or a
                              // sector's relative 1e-10 cut-off met a value within two decades of it
  double cut_gap = 1.0;       // (D-th - (D+1)-th singular value) / |psi|; 1 when nothing was cut
};

// BlockTensor::svd (src/block_tensor_inst.cpp:501-637)
template <class S>
SvdStats block_svd(Ctx& c, const BTensor<S>& psi, BTensor<S>& tu, double p1, BTensor<S>& tv, double p2,
                   int max_dcut, std::vector<double>* wout);

struct Timers {
  double lanczos = 0, env = 0, svd = 0, prep = 0;   // host wall time of each phase
  long long matvecs = 0;
  double heff_flops = 0;
  double svd_kernel = 0;        // device time of the Jacobi sweep kernels (s)
  long long svd_sweeps = 0;     // Jacobi sweeps, summed over the truncations
  double plan = 0;              // host wall time of building H_eff plans (part of lanczos)
};

template <class S>
class Chain {
 public:
  Chain(Ctx& c, int lx, int ly, int bondd, int physpn, int totspin, int open, double J2);
  void do_idmrg();
  void prepare_sweep();
  void sweep();
  double energy() const { return gs_enr; }
  // Dz (S_a x S_b)_z on every J1 bond a < b (U(1), complex only; before iDMRG)
  void set_dm(double d);
  // the k-th excited state (the constructor's max_exci, src/dmrg_inst.cpp:64-112):
  // read_mps then loads this state's files (index k) and the lower states' (0 .. k-1,
  // into orth) with their energies, and the sweeps add the overlap environments and
  // the penalty (before read_mps; U(1) and SU(2))
  void set_excited(int k);

  // building blocks (public for the frozen-problem API and tests)
  // flag (real environments of an excited-state chain): also the lower states
  // projected on sites i+1, i+2 (from the left) or i-2, i-1 (from the right)
  void prepare_site_operator_from_left(int i, bool real_env, int flag = 0);
  void prepare_site_operator_from_right(int i, bool real_env, int flag = 0);
  void prepare_input_vector(int il, int ir, BTensor<S>& vec);
  void prepare_input_vector_initial(int il, int ir, BTensor<S>& vec);
  HeffPlan<S> heff_plan(int il, int ir, const BTensor<S>& vec, bool tune = false);
  void lanczos_solve_eigenvector(int il, int ir, BTensor<S>& vec);
  void wavefunc_transformation(int i, int dir);
  // DMRG::read_mps / save_mps2 checkpoint format (src/dmrg_inst.cpp:947-1079)
  bool read_mps(const std::string& dir, int bond_read);
  bool read_state(const std::string& dir, int bond_read, int idx, std::vector<BTensor<S>>& out);
  void save_mps(const std::string& dir) const;
  // DMRG::save_ww / read_ww / save_enr / read_enr (src/dmrg_inst.cpp:993-1030, 1145-1177)
  void save_ww(const std::string& dir) const;
  void read_ww(const std::string& dir, int read1);
  void save_enr(const std::string& dir) const;
  void read_enr(const std::string& dir, int read1);
  // the two-site problem at bond (il, il+1): psi from the current site tensors and
  // the H_eff plan of DMRG::hamiltonian_vector_multiplication_idmrg
  HeffPlan<S> freeze(int il, BTensor<S>& psi);
  // the same problem written as text-structure + binary-data files (one pair per tensor)
  void export_problem(int il, const BTensor<S>& psi, const std::string& dir) const;

  Ctx& c;
  int lx, ly, ns, bondd, physpn, totspin, nfree = 2;
  int max_dcut;
  std::vector<std::vector<int>> hmap, fll, frr;
  std::vector<double> coup;
  double dz = 0.0;            // DM coupling on J1 bonds (set_dm)
  std::vector<BTensor<S>> uu, hh;
  std::vector<std::vector<BTensor<S>>> opr;
  std::array<BTensor<S>, 2> sigma;
  double gs_enr = 0.0;
  // excited states (set_excited): exci lower states orth[j][i], their overlap
  // environments with uu ovlp[j][i] (site tensors of the lower state projected on
  // the current basis at the two sites of a step), their energies and their
  // projections on the current two-site basis (the penalty vectors)
  int exci = 0;
  std::vector<std::vector<BTensor<S>>> orth, ovlp;
  std::vector<double> low_enr;
  std::vector<BTensor<S>> overlapvec;
  // singular values of the truncations, laid out as the reference's ww array:
  // each truncation overwrites its first n values (kept, then discarded)
  std::vector<double> ww;
  double last_discarded = 0.0;
  int near_ties = 0;          // truncations whose cut fell inside a near-degenerate pair
  int stop_ties = 0;          // truncations whose cut gap is below 10 sqrt(Lanczos ov_tol) |psi|
  std::vector<int> bond_flags;  // per bond (site il of the pair): flags of its last truncation,
                                // 1 a rounding tie (near_ties), 2 a stop-test tie
  // Lanczos settings (reference constants at src/dmrg_inst.cpp:267,1289,1338)
  int mlanc_max = 40;
  int prec = PREC_FP64;
  Timers timers;
  std::mt19937_64 rng{42};  // the reference's generator (src/dense_inst.cpp:23-24)
  std::uniform_real_distribution<double> dist{-1.0, 1.0};
  std::vector<std::string> log;

 private:
  void random_init(BTensor<S>& t);
  void init_local_operators();
  void svd_step(BTensor<S>& vec, int il, int ir, double p1, double p2);
  void set_penalty(HeffPlan<S>& H, const BTensor<S>& vec);
  void add_coupled(BTensor<S>& op, const BTensor<S>& src, int a, int b);
};

}  // namespace sadmrg
