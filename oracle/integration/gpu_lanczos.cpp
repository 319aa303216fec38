// gpu_lanczos.cpp -- the reference's own DMRG sweep with its Lanczos solve on the GPU.
//
// Test infrastructure: it shows the drop-in boundary compiled against the
// reference.  This translation unit includes the reference's headers and gives
// DMRG<Scalar,Sym>::lanczos_solve_eigenvector_idmrg (src/dmrg_inst.cpp:264-279)
// a new body that goes through include/sadmrg.h:
//   * the operator set of DMRG::hamiltonian_vector_multiplication_idmrg
//     (src/dmrg_inst.cpp:309-351: for every left operator j the right operators
//     k it pairs with, summed with their couplings) and the block Hamiltonians
//     are handed over as sadmrg_tensor_desc views of the reference's
//     BlockTensors and planned (sadmrg_heff_plan);
//   * Lanczos runs on the GPU (sadmrg_heff_lanczos, FP64 or split precision)
//     with the reference's mlanc and stop test;
//   * the Ritz vector is copied back into vec's blocks and gs_enr[exci] is set.
// The new bodies are strong symbols with the method's own linker names; the
// linker takes them over the weak ones of the reference's explicit
// instantiations, so the reference's unmodified sweep() (src/dmrg_inst.cpp:874-943)
// calls them (the driver counts the calls).
//
// Driver: reads a save_mps2 checkpoint (read_mps + prepare_sweep), sets up open
// boundaries as the harness does, runs N sweeps and prints
//   SWEEP s E <energy>     BONDS s site i q:d ...     GPU_LANCZOS_CALLS n
#include <omp.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

// the driver below reads the chain's members the way the harness does
#define private public
#define protected public
#include "dmrg.hpp"
#include "cgc_tables.hpp"
#undef private
#undef protected
#include "../shims/lanczos_knobs.h"
#include "../../include/sadmrg.h"

int max_dcut = 64;
int psize = 1;
int myrank = 0;
CGCTables* g_cgc_tables = nullptr;
int ref_lanczos_mlanc = 40;
double ref_lanczos_check = 1e-8;

static sadmrg_handle* g_gpu = nullptr;
static int g_gpu_calls = 0;
static int g_gpu_prec = SADMRG_PREC_FP64;

// BlockTensor<Scalar,Sym> -> sadmrg_tensor_desc (the arrays must outlive the call)
template <class Scalar, class Sym>
struct Desc {
  std::vector<int> dir, nmom, q, d;
  std::vector<long long> blocks;
  std::vector<Scalar> data;
  sadmrg_tensor_desc view{};
  explicit Desc(BlockTensor<Scalar, Sym>& t) {
    const int nb = t.get_nbond();
    for (int b = 0; b < nb; ++b) {
      dir.push_back(t.get_bonddir(b));
      nmom.push_back(t.get_nmoment(b));
      for (int k = 0; k < t.get_nmoment(b); ++k) {
        q.push_back(t.get_angularmoment(b, k));
        d.push_back(t.get_bonddim(b, k));
      }
    }
    std::vector<int> angm(nb), bdim(nb);
    for (int i = 0; i < t.get_nten(); ++i) {
      if (!t.get_tensor_argument(i, angm.data(), bdim.data())) continue;
      Dense<Scalar>* blk = t.get_data_block(i);
      if (blk->is_null()) continue;
      blocks.push_back(i);
      data.insert(data.end(), blk->getptr(), blk->getptr() + blk->get_nelem());
    }
    view = {nb, t.get_locspin(), dir.data(), nmom.data(), q.data(), d.data(), (int)blocks.size(), blocks.data(),
            data.data()};
  }
};

static void check(int rc, const char* what) {
  if (rc != SADMRG_OK) {
    std::cerr << what << " failed (" << rc << "): " << sadmrg_last_error(g_gpu) << "\n";
    std::exit(3);
  }
}

// the body every variant below shares; the chain's members are passed in
template <class Scalar, class Sym>
static double gpu_solve(int il, int ir, BlockTensor<Scalar, Sym>& vec, int ns, BlockTensor<Scalar, Sym>* hh,
                        BlockTensor<Scalar, Sym>** opr, int** hmap, const double* coup) {
  using TensorType = BlockTensor<Scalar, Sym>;
  // operator set of hamiltonian_vector_multiplication_idmrg (src/dmrg_inst.cpp:309-351)
  std::vector<TensorType> sums;
  std::vector<TensorType*> fixed;
  int m1, m4;
  if (il < ns / 2) { m1 = il + 1; m4 = ns - ir; }
  else { m1 = ns - ir; m4 = il + 1; }
  for (int m0 = 0; m0 < m1; ++m0) {
    int j = 0, k = 0;
    if (il < ns / 2) j = m0;
    else k = ir + m0;
    TensorType op;
    for (int m = 0; m < m4; ++m) {
      if (il < ns / 2) k = ir + m;
      else j = m;
      if (hmap[j][k] > 0) {
        TensorType ht = (il < ns / 2) ? opr[ir][k] : opr[il][j];
        ht *= coup[hmap[j][k]];
        if (op.is_null()) op = ht;
        else op += ht;
      }
    }
    if (op.is_null()) continue;
    TensorType* f = (il < ns / 2) ? &opr[il][j] : &opr[ir][k];
    if (f->is_null()) continue;
    sums.push_back(op);
    fixed.push_back(f);
  }
  std::vector<Desc<Scalar, Sym>> ops;
  ops.reserve(2 * sums.size());
  std::vector<int> op1, op2;
  for (size_t t = 0; t < sums.size(); ++t) {
    ops.emplace_back(*fixed[t]);
    ops.emplace_back(sums[t]);
    const int fi = (int)ops.size() - 2, si = (int)ops.size() - 1;
    op1.push_back(il < ns / 2 ? fi : si);
    op2.push_back(il < ns / 2 ? si : fi);
  }
  std::vector<sadmrg_tensor_desc> v;
  for (auto& o : ops) v.push_back(o.view);
  Desc<Scalar, Sym> psi(vec);
  Desc<Scalar, Sym>* hl = hh[il].is_null() ? nullptr : new Desc<Scalar, Sym>(hh[il]);
  Desc<Scalar, Sym>* hr = hh[ir].is_null() ? nullptr : new Desc<Scalar, Sym>(hh[ir]);
  check(sadmrg_heff_plan(g_gpu, &psi.view, hl ? &hl->view : nullptr, hr ? &hr->view : nullptr, (int)v.size(),
                         v.data(), (int)op1.size(), op1.data(), op2.data()),
        "sadmrg_heff_plan");
  // the reference's Lanczos length (src/dmrg_inst.cpp:267-270) and stop test (:1338)
  int ndata = 0, ncgc = 0;
  vec.get_nelement(ndata, ncgc);
  int mlanc = ref_lanczos_mlanc;
  if (mlanc > ndata) mlanc = ndata + 1;
  if (mlanc < 2) mlanc = 2;
  check(sadmrg_set_lanczos_tol(g_gpu, ref_lanczos_check), "sadmrg_set_lanczos_tol");
  double E = 0.0;
  int nmv = 0;
  check(sadmrg_heff_lanczos(g_gpu, psi.data.data(), mlanc, g_gpu_prec, &E, &nmv), "sadmrg_heff_lanczos");
  // the Ritz vector back into vec's blocks (psi's block order)
  size_t off = 0;
  for (long long b : psi.blocks) {
    Dense<Scalar>* blk = vec.get_data_block((int)b);
    std::copy(psi.data.begin() + off, psi.data.begin() + off + blk->get_nelem(), blk->getptr());
    off += blk->get_nelem();
  }
  delete hl;
  delete hr;
  ++g_gpu_calls;
  return E;
}

// The new bodies carry the linker names (Itanium C++ ABI) of the member
// DMRG<S, Sym>::lanczos_solve_eigenvector_idmrg(int, int, TensorType&), whose
// first argument is the object.  They cannot be written as explicit
// specializations: dmrg.hpp declares `extern template class DMRG<double,
// SU2Symmetry>` (and the complex one), after which a specialization is ill-formed.
#define GPU_LANCZOS(S, SYM, NAME)                                                                      \
  void gpu_lanczos_##NAME(DMRG<S, SYM>* self, int il, int ir, BlockTensor<S, SYM>& vec) __asm__(#NAME); \
  void gpu_lanczos_##NAME(DMRG<S, SYM>* self, int il, int ir, BlockTensor<S, SYM>& vec) {              \
    self->gs_enr[self->exci] =                                                                         \
        gpu_solve<S, SYM>(il, ir, vec, self->ns, self->hh, self->opr, self->hmap, self->coup);         \
  }
GPU_LANCZOS(double, U1Symmetry, _ZN4DMRGId10U1SymmetryE31lanczos_solve_eigenvector_idmrgEiiR11BlockTensorIdS0_E)
GPU_LANCZOS(double, SU2Symmetry, _ZN4DMRGId11SU2SymmetryE31lanczos_solve_eigenvector_idmrgEiiR11BlockTensorIdS0_E)
GPU_LANCZOS(dcmplex, U1Symmetry,
            _ZN4DMRGISt7complexIdE10U1SymmetryE31lanczos_solve_eigenvector_idmrgEiiR11BlockTensorIS1_S2_E)
GPU_LANCZOS(dcmplex, SU2Symmetry,
            _ZN4DMRGISt7complexIdE11SU2SymmetryE31lanczos_solve_eigenvector_idmrgEiiR11BlockTensorIS1_S2_E)

// ---- driver ----------------------------------------------------------------
// open boundaries and J2 on the constructor's periodic lattice (the harness's set-up)
static void open_lattice(int** hmap, int** fll, int** frr, double* coup, int ns, int lx, int ly, double J2) {
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < ns; ++j) hmap[i][j] = 0;
  auto site = [&](int x, int y) { return (x % 2 == 0) ? x * ly + y : x * ly + (ly - 1 - y); };
  for (int i = 0; i < ns; ++i) {
    const int x1 = i / ly, y1 = (x1 % 2 == 0) ? i % ly : ly - 1 - (i % ly);
    for (int k = 0; k < 2; ++k) {
      int x2 = x1, y2 = y1;
      if (k == 0) { x2 = x1 + 1; if (x2 >= lx) continue; }
      else { y2 = y1 + 1; if (y2 >= ly) continue; }
      const int j = site(x2, y2);
      if (i != j) { hmap[i][j] = 1; hmap[j][i] = 1; }
    }
  }
  for (int i = 0; i <= ns / 2; ++i) coup[i] = 0.0;
  coup[1] = 1.0;
  if (J2 != 0.0) {
    for (int i = 0; i + 2 < ns; ++i) { hmap[i][i + 2] = 2; hmap[i + 2][i] = 2; }
    coup[2] = J2;
  }
  for (int i = 0; i < ns; ++i) {
    for (int j = 0; j < ns; ++j) { fll[i][j] = 0; frr[i][j] = 0; }
    for (int j = 0; j < i; ++j)
      for (int k = i + 1; k < ns; ++k)
        if (hmap[j][k] != 0) fll[i][j] = 1;
    for (int j = i + 1; j < ns; ++j)
      for (int k = 0; k < i; ++k)
        if (hmap[j][k] != 0) frr[i][j] = 1;
  }
}

struct Opts {
  int sym = 1, cplx = 0, lx = 1, ly = 12, D = 16, sweeps = 2, threads = 1;
  double J2 = 0.0;
  std::string read;
};

template <class S, class Sym>
static int run(const Opts& o) {
  max_dcut = o.D;
  // the reference sizes its per-thread buffers by psize: OpenMP must use that many threads
  psize = o.threads;
  omp_set_num_threads(o.threads);
  std::streambuf* saved = std::cout.rdbuf();
  std::ostringstream sink;
  std::cout.rdbuf(sink.rdbuf());
  DMRG<S, Sym> chain(o.lx, o.ly, o.D, 1, 0, 0);
  std::cout.rdbuf(saved);
  open_lattice(chain.hmap, chain.fll, chain.frr, chain.coup, chain.ns, chain.lx, chain.ly, o.J2);
  delete[] chain.ww[0];
  chain.ww[0] = new double[64 * o.D + 4096]();   // room for every singular value BlockTensor::svd writes
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd))) return 3;
  if (chdir(o.read.c_str()) != 0) { std::cerr << "cannot enter " << o.read << "\n"; return 3; }
  std::cout.rdbuf(sink.rdbuf());
  const bool ok = chain.read_mps(o.D);
  if (ok) chain.prepare_sweep();
  std::cout.rdbuf(saved);
  if (!ok) { std::cerr << "read_mps failed\n"; return 3; }
  const std::string sw = std::string(cwd) + "/sweep_files";   // sweep() writes its checkpoint files here
  mkdir(sw.c_str(), 0755);
  if (chdir(sw.c_str()) != 0) return 3;
  for (int s = 0; s < o.sweeps; ++s) {
    std::cout.rdbuf(sink.rdbuf());
    chain.sweep();
    std::cout.rdbuf(saved);
    sink.str("");
    std::cout << std::setprecision(16) << "SWEEP " << s << " E " << chain.get_enr() << "\n";
    for (int i = 0; i < chain.ns; ++i) {
      BlockTensor<S, Sym>& u = chain.uu[i];
      if (u.get_nbond() < 3) continue;
      std::cout << "BONDS " << s << " site " << i;
      for (int k = 0; k < u.get_nmoment(2); ++k)
        std::cout << " " << u.get_angularmoment(2, k) << ":" << u.get_bonddim(2, k);
      std::cout << "\n";
    }
  }
  if (chdir(cwd) != 0) return 3;
  std::cout << "GPU_LANCZOS_CALLS " << g_gpu_calls << "\n";
  return 0;
}

int main(int argc, char** argv) {
  Opts o;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto nxt = [&]() { return std::string(argv[++i]); };
    if (a == "-sym") o.sym = nxt() == "su2" ? 1 : 0;
    else if (a == "-cplx") o.cplx = std::stoi(nxt());
    else if (a == "-L") { o.lx = 1; o.ly = std::stoi(nxt()); }
    else if (a == "-lx") o.lx = std::stoi(nxt());
    else if (a == "-ly") o.ly = std::stoi(nxt());
    else if (a == "-d") o.D = std::stoi(nxt());
    else if (a == "-J2") o.J2 = std::stod(nxt());
    else if (a == "-sweeps") o.sweeps = std::stoi(nxt());
    else if (a == "-read") o.read = nxt();
    else if (a == "-mlanc") ref_lanczos_mlanc = std::stoi(nxt());
    else if (a == "-lanc_check") ref_lanczos_check = std::stod(nxt());
    else if (a == "-prec") g_gpu_prec = std::stoi(nxt());
    else if (a == "-threads") o.threads = std::stoi(nxt());
    else { std::cerr << "unknown option " << a << "\n"; return 2; }
  }
  if (o.read.empty()) { std::cerr << "-read <checkpoint dir> is required\n"; return 2; }
  if (sadmrg_create(o.sym, o.cplx, 0, &g_gpu) != SADMRG_OK) { std::cerr << "sadmrg_create failed\n"; return 3; }
  int rc;
  if (o.sym == 0 && o.cplx == 0) rc = run<double, U1Symmetry>(o);
  else if (o.sym == 0) rc = run<dcmplex, U1Symmetry>(o);
  else if (o.cplx == 0) rc = run<double, SU2Symmetry>(o);
  else rc = run<dcmplex, SU2Symmetry>(o);
  sadmrg_destroy(g_gpu);
  return rc;
}
