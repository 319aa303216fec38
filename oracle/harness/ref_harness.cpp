// ref_harness.cpp -- driver for the reference CPU build (test infrastructure only).
//
// Compiled against the reference's own headers and sources (built by
// oracle/Makefile into oracle/_ref/).  It never changes the reference's
// arithmetic; it only sets up the cases the reference's mains cannot express
// and dumps what the reference computes so the oracle and the GPU path can be
// checked against it.
//
// Harness-only set-up (none edits a reference file):
//   * open boundaries / J2: the constructor hard-codes a periodic nearest-
//     neighbour hmap (src/dmrg_inst.cpp:121-160); we rebuild hmap, coup, fll and
//     frr after construction with the same loops (src/dmrg_inst.cpp:163-176).
//   * U(1) D cap: the U1 main never sets max_dcut (main/main_dmrg_u1_real.cpp:50);
//     here max_dcut = D for both symmetries.
//   * max_angm: the constructor builds CGC tables with max_angm = 20
//     (src/dmrg_inst.cpp:181); when -maxangm is larger the tables are rebuilt.
//   * ww buffer: BlockTensor::svd writes every singular value into a bondd-long
//     array (src/block_tensor_inst.cpp:579-602 vs src/dmrg_inst.cpp:84); we give
//     it room for all of them.
//   * fixed sweep count, no early stop.
//   * Lanczos settings: -mlanc / -lanc_check set the two constants the
//     reference hard-codes (src/dmrg_inst.cpp:267 mlanc = 40, :1338 stop at
//     |<v|Hv>|/|Hv| within 1e-8 of 1); oracle/Makefile compiles dmrg_inst.cpp
//     with those constants read from the globals below, defaults unchanged.
//   * -sweepdir: the directory sweep() writes its checkpoint files to
//     (save_mps2 / save_ww / save_enr, src/dmrg_inst.cpp:940-942).
// Private members are reached with the usual access-specifier override.
#include <omp.h>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <sstream>
#include <vector>
#include <map>

#define private public
#define protected public
#include "dmrg.hpp"
#include "cgc_tables.hpp"
#undef private
#undef protected
#include "../shims/lanczos_knobs.h"

int max_dcut = 64;
int psize = 1;
int myrank = 0;
CGCTables* g_cgc_tables = nullptr;
int ref_lanczos_mlanc = 40;        // src/dmrg_inst.cpp:267
double ref_lanczos_check = 1e-8;   // src/dmrg_inst.cpp:1338
void makeup_clebsch_gordan_coefficient_tensors(int physpn, int max_angm, CGCTables& t);

struct Opts;
template <class S, class Sym> static int run_load(const Opts& o);

struct Opts {
  int sym = 0;       // 0 = U1, 1 = SU2
  int cplx = 0;      // 0 = double, 1 = dcmplex
  int lx = 1, ly = 8;
  int D = 32, sec = 0, sweeps = 2, threads = 1, maxangm = 0, open = 1;
  double J2 = 0.0;
  std::string dump;  // directory: dump the centre two-site problem there
  std::string save;  // directory: save_mps2 after iDMRG (checkpoint files)
  std::string read;  // directory: read_mps + prepare_sweep instead of iDMRG
  int bench_heff = 0;  // time this many H*v calls on the centre problem
  std::string load;    // directory with an exported two-site problem (time / check H*v on it)
  int quiet = 1;
  int mlanc = 40;           // Lanczos length (reference: 40)
  double lanc_check = 1e-8; // Lanczos stop test (reference: 1e-8)
  std::string sweepdir = "/tmp";
  int exci = 0;             // excited state: DMRG(..., max_exci = exci); with -read, read_mps(D, D)
                            // loads this state's files (index exci) and the lower states' (0..exci-1)
};

template <class S, class Sym>
static void dump_tensor(const std::string& dir, const std::string& name, BlockTensor<S, Sym>& t) {
  std::ofstream ft(dir + "/" + name + ".txt");
  std::ofstream fb(dir + "/" + name + ".bin", std::ios::binary);
  int nb = t.get_nbond();
  ft << "nbond " << nb << " locspin " << t.get_locspin() << " nten " << t.get_nten() << "\n";
  for (int b = 0; b < nb; ++b) {
    int nm = t.get_nmoment(b);
    ft << "bond " << b << " dir " << t.get_bonddir(b) << " nmom " << nm << " q";
    for (int k = 0; k < nm; ++k) ft << " " << t.get_angularmoment(b, k);
    ft << " d";
    for (int k = 0; k < nm; ++k) ft << " " << t.get_bonddim(b, k);
    ft << "\n";
  }
  long off = 0;
  std::vector<int> angm(nb > 0 ? nb : 1), bdim(nb > 0 ? nb : 1), cdim(nb > 0 ? nb : 1);
  for (int i = 0; i < t.get_nten(); ++i) {
    if (!t.get_tensor_argument(i, angm.data(), bdim.data(), cdim.data())) continue;
    if (t.data_blocks[i].check_null()) continue;
    Dense<S>& d = t.data_blocks[i];
    ft << "block " << i << " q";
    for (int b = 0; b < nb; ++b) ft << " " << angm[b];
    ft << " d";
    for (int b = 0; b < d.get_nbond(); ++b) ft << " " << d.get_bonddim(b);
    ft << " off " << off << " n " << d.get_nelem() << "\n";
    fb.write(reinterpret_cast<const char*>(d.getptr()), sizeof(S) * d.get_nelem());
    off += d.get_nelem();
  }
}

template <class S, class Sym>
static void print_bonds(DMRG<S, Sym>& c, const char* tag) {
  for (int i = 0; i < c.ns; ++i) {
    BlockTensor<S, Sym>& u = c.uu[i];
    if (u.get_nbond() < 3) continue;
    std::cout << tag << " site " << i;
    int nm = u.get_nmoment(2);
    for (int k = 0; k < nm; ++k) std::cout << " " << u.get_angularmoment(2, k) << ":" << u.get_bonddim(2, k);
    std::cout << "\n";
  }
}

template <class S, class Sym>
static void patch_geometry(DMRG<S, Sym>& c, const Opts& o) {
  int ns = c.ns, lx = c.lx, ly = c.ly;
  for (int i = 0; i < ns; ++i)
    for (int j = 0; j < ns; ++j) c.hmap[i][j] = 0;
  auto site = [&](int x, int y) { return (x % 2 == 0) ? x * ly + y : x * ly + (ly - 1 - y); };
  for (int i = 0; i < ns; ++i) {
    int x1 = i / ly, y1 = (x1 % 2 == 0) ? i % ly : ly - 1 - (i % ly);
    for (int k = 0; k < 2; ++k) {
      int x2 = x1, y2 = y1;
      if (k == 0) { x2 = x1 + 1; if (x2 >= lx) { if (o.open) continue; x2 %= lx; } }
      else        { y2 = y1 + 1; if (y2 >= ly) { if (o.open) continue; y2 %= ly; } }
      int j = site(x2, y2);
      if (i != j) { c.hmap[i][j] = 1; c.hmap[j][i] = 1; }
    }
  }
  for (int i = 0; i <= ns / 2; ++i) c.coup[i] = 0.0;
  c.coup[1] = 1.0;
  if (o.J2 != 0.0) {
    for (int i = 0; i + 2 < ns; ++i) { c.hmap[i][i + 2] = 2; c.hmap[i + 2][i] = 2; }
    c.coup[2] = o.J2;
  }
  for (int i = 0; i < ns; ++i) {
    for (int j = 0; j < ns; ++j) { c.fll[i][j] = 0; c.frr[i][j] = 0; }
    for (int j = 0; j < i; ++j)
      for (int k = i + 1; k < ns; ++k)
        if (c.hmap[j][k] != 0) c.fll[i][j] = 1;
    for (int j = i + 1; j < ns; ++j)
      for (int k = 0; k < i; ++k)
        if (c.hmap[j][k] != 0) c.frr[i][j] = 1;
  }
}

template <class S, class Sym>
static int run(const Opts& o) {
  max_dcut = o.D;
  psize = o.threads;
  omp_set_num_threads(o.threads);
  std::streambuf* saved = std::cout.rdbuf();
  std::ostringstream sink;
  auto mute = [&]() { if (o.quiet) std::cout.rdbuf(sink.rdbuf()); };
  auto unmute = [&]() { std::cout.rdbuf(saved); sink.str(""); };

  mute();
  DMRG<S, Sym> chain(o.lx, o.ly, o.D, 1, o.sec, o.exci);
  if constexpr (Sym::has_cgc) {
    if (o.maxangm > 20) {
      delete g_cgc_tables;
      g_cgc_tables = new CGCTables();
      makeup_clebsch_gordan_coefficient_tensors(1, o.maxangm, *g_cgc_tables);
    }
  }
  unmute();
  patch_geometry(chain, o);
  // room for every singular value BlockTensor::svd may write
  int wlen = 64 * o.D + 4096;
  for (int e = 0; e <= o.exci; ++e) {
    delete[] chain.ww[e];
    chain.ww[e] = new double[wlen]();
  }

  auto t0 = std::chrono::steady_clock::now();
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd))) cwd[0] = 0;
  if (!o.read.empty()) {
    // DMRG::read_mps + prepare_sweep (src/dmrg_inst.cpp:1031-1079, 808-854)
    if (chdir(o.read.c_str()) != 0) { std::cerr << "cannot enter " << o.read << "\n"; return 3; }
    mute();
    // an excited state: DMRG::read_mps(read1, read2) (src/dmrg_inst.cpp:1081-1140) also
    // loads the lower states into orth and their energies (read_enr)
    bool ok = o.exci > 0 ? chain.read_mps(o.D, o.D) : chain.read_mps(o.D);
    if (ok) chain.prepare_sweep();
    unmute();
    if (chdir(cwd) != 0) return 3;
    if (!ok) { std::cerr << "read_mps failed in " << o.read << "\n"; return 3; }
  } else {
    mute();
    chain.do_idmrg();
    unmute();
  }
  if (!o.save.empty()) {
    mkdir(o.save.c_str(), 0755);
    if (chdir(o.save.c_str()) != 0) return 3;
    chain.save_mps2(0);
    if (chdir(cwd) != 0) return 3;
  }
  auto t1 = std::chrono::steady_clock::now();
  std::cout << std::setprecision(16) << "IDMRG E " << chain.get_enr() << " seconds "
            << std::chrono::duration<double>(t1 - t0).count() << "\n";
  print_bonds(chain, "BONDS -1");
  for (int s = 0; s < o.sweeps; ++s) {
    auto a = std::chrono::steady_clock::now();
    mute();
    // sweep() writes its checkpoint files to the working directory
    mkdir(o.sweepdir.c_str(), 0755);
    if (chdir(o.sweepdir.c_str()) != 0) return 3;
    chain.sweep();
    if (chdir(cwd) != 0) return 3;
    unmute();
    auto b = std::chrono::steady_clock::now();
    std::cout << std::setprecision(16) << "SWEEP " << s << " E " << chain.get_enr() << " seconds "
              << std::chrono::duration<double>(b - a).count() << "\n";
    std::string tag = "BONDS " + std::to_string(s);
    print_bonds(chain, tag.c_str());
  }
  std::cout.flush();

  if (!o.dump.empty() || o.bench_heff > 0) {
    // the first step of the left-moving half sweep (src/dmrg_inst.cpp:880-897)
    int i = chain.ns / 2, il = i - 2, ir = i - 1;
    BlockTensor<S, Sym> vec, out;
    const std::string& dd = o.dump;
    if (!dd.empty()) {
      mkdir(dd.c_str(), 0755);
      dump_tensor(dd, "uu_i_before", chain.uu[i]);
      dump_tensor(dd, "hh_ip1", chain.hh[i + 1]);
      for (int k = 0; k < chain.ns; ++k)
        if (!chain.opr[i + 1][k].is_null()) dump_tensor(dd, "opr_ip1_" + std::to_string(k), chain.opr[i + 1][k]);
    }
    mute();
    chain.wavefunc_transformation(i - 1, 1);
    chain.prepare_site_operator_from_right(i, 1);
    unmute();
    if (!dd.empty()) {
      dump_tensor(dd, "uu_i", chain.uu[i]);
      dump_tensor(dd, "hh_i", chain.hh[i]);
      for (int k = 0; k < chain.ns; ++k)
        if (!chain.opr[i][k].is_null()) dump_tensor(dd, "opr_i_" + std::to_string(k), chain.opr[i][k]);
      dump_tensor(dd, "uu_il", chain.uu[il]);
      dump_tensor(dd, "uu_ir", chain.uu[ir]);
      dump_tensor(dd, "hh_ilm1", chain.hh[il - 1]);
      for (int k = 0; k < chain.ns; ++k)
        if (!chain.opr[il - 1][k].is_null()) dump_tensor(dd, "opr_ilm1_" + std::to_string(k), chain.opr[il - 1][k]);
    }
    mute();
    chain.prepare_input_vector(il, ir, vec);
    chain.prepare_site_operator_from_left(il);
    chain.prepare_site_operator_from_right(ir);
    unmute();
    vec.normalize_vector();
    if (!dd.empty()) {
      dump_tensor(dd, "psi", vec);
      dump_tensor(dd, "hh_il", chain.hh[il]);
      dump_tensor(dd, "hh_ir", chain.hh[ir]);
      for (int k = 0; k < chain.ns; ++k) {
        if (!chain.opr[il][k].is_null()) dump_tensor(dd, "opr_il_" + std::to_string(k), chain.opr[il][k]);
        if (!chain.opr[ir][k].is_null()) dump_tensor(dd, "opr_ir_" + std::to_string(k), chain.opr[ir][k]);
      }
    }
    mute();
    chain.hamiltonian_vector_multiplication_idmrg(il, ir, vec, out);
    unmute();
    if (!dd.empty()) {
      dump_tensor(dd, "hpsi", out);
      std::ofstream fm(dd + "/meta.txt");
      fm << std::setprecision(17);
      fm << "sym " << o.sym << " cplx " << o.cplx << " ns " << chain.ns << " lx " << chain.lx << " ly " << chain.ly
         << " D " << o.D << " sec " << o.sec << " il " << il << " ir " << ir << " J2 " << o.J2 << " open " << o.open
         << " maxangm " << (o.maxangm > 20 ? o.maxangm : 20) << "\n";
      fm << "coup";
      for (int k = 0; k <= chain.ns / 2; ++k) fm << " " << chain.coup[k];
      fm << "\n";
      for (int a = 0; a < chain.ns; ++a)
        for (int b = 0; b < chain.ns; ++b)
          if (chain.hmap[a][b]) fm << "hmap " << a << " " << b << " " << chain.hmap[a][b] << "\n";
      // Lanczos on the same start vector, then the SVD truncation that follows
      BlockTensor<S, Sym> v2 = vec;
      mute();
      chain.lanczos_solve_eigenvector_idmrg(il, ir, v2);
      unmute();
      fm << "lanczos_E " << chain.gs_enr[0] << "\n";
      dump_tensor(dd, "psi_gs", v2);
      BlockTensor<S, Sym> ul = chain.uu[il], ur = chain.uu[ir];
      for (int k = 0; k < wlen; ++k) chain.ww[0][k] = 0.0;
      mute();
      v2.svd(ul, 1.0, ur, 0.0, chain.ww[0]);
      unmute();
      dump_tensor(dd, "svd_u", ul);
      dump_tensor(dd, "svd_v", ur);
      fm << "svd_w";
      for (int k = 0; k < wlen && chain.ww[0][k] != 0.0; ++k) fm << " " << chain.ww[0][k];
      fm << "\n";
    }
    if (o.bench_heff > 0) {
      auto a = std::chrono::steady_clock::now();
      mute();
      for (int r = 0; r < o.bench_heff; ++r) chain.hamiltonian_vector_multiplication_idmrg(il, ir, vec, out);
      unmute();
      auto b = std::chrono::steady_clock::now();
      std::cout << std::setprecision(10) << "BENCH_HEFF calls " << o.bench_heff << " seconds "
                << std::chrono::duration<double>(b - a).count() << " threads " << o.threads << "\n";
    }
  }
  return 0;
}

// ---- exported two-site problem ---------------------------------------------
// Reads the <name>.txt / <name>.bin pairs written by the GPU library's problem
// export into the reference's own BlockTensors and runs the reference's
// DMRG::hamiltonian_vector_multiplication_idmrg on them.
template <class S, class Sym>
static bool load_tensor(const std::string& dir, const std::string& name, BlockTensor<S, Sym>& t, bool psi) {
  std::ifstream ft(dir + "/" + name + ".txt");
  if (!ft) return false;
  std::string line, w;
  int nb = 0, ls = 0;
  // BondType has no copy constructor: keep the raw labels and set the bonds in place
  std::vector<std::vector<int>> bq, bdm;
  std::vector<int> bdir;
  struct B { long idx; std::vector<int> dims; long off, n; };
  std::vector<B> blocks;
  while (std::getline(ft, line)) {
    std::istringstream is(line);
    is >> w;
    if (w == "nbond") { long nten; std::string a, b; is >> nb >> a >> ls >> b >> nten; }
    else if (w == "bond") {
      int bi, dir, nm; std::string a, c, q;
      is >> bi >> a >> dir >> c >> nm >> q;
      std::vector<int> qs(nm), ds(nm);
      for (int k = 0; k < nm; ++k) is >> qs[k];
      is >> q;
      for (int k = 0; k < nm; ++k) is >> ds[k];
      bq.push_back(qs);
      bdm.push_back(ds);
      bdir.push_back(dir);
    } else if (w == "block") {
      B b; std::string x;
      is >> b.idx >> x;
      for (int k = 0; k < nb; ++k) { int qq; is >> qq; }
      is >> x;
      b.dims.resize(nb);
      for (int k = 0; k < nb; ++k) is >> b.dims[k];
      is >> x >> b.off >> x >> b.n;
      blocks.push_back(b);
    }
  }
  typename Sym::BondType* bonds = new typename Sym::BondType[nb];
  for (int b = 0; b < nb; ++b) bonds[b].set(bdir[b], (int)bq[b].size(), bq[b].data(), bdm[b].data());
  typename Sym::StructType st;
  st.set_struct(nb, ls, bonds);
  delete[] bonds;
  t.set(st, nullptr, nullptr);
  std::ifstream fb(dir + "/" + name + ".bin", std::ios::binary);
  fb.seekg(0, std::ios::end);
  const long nbytes = fb.tellg();
  fb.seekg(0);
  std::vector<S> data(nbytes / sizeof(S));
  fb.read(reinterpret_cast<char*>(data.data()), nbytes);
  for (auto& b : blocks) t.data_blocks[b.idx].copy(nb, b.dims.data(), data.data() + b.off);
  if constexpr (Sym::has_cgc) {
    if (psi) {  // the two-site vector carries singlet CGC blocks (makeup_input_vector)
      std::vector<int> angm(nb), bdim(nb);
      for (int i = 0; i < t.nten; ++i)
        if (t.cgc.get_tensor_argument(i, angm.data(), bdim.data())) t.cgc_blocks[i].make_singlet(angm[0]);
    }
  }
  return true;
}

template <class S, class Sym>
static int run_load(const Opts& o) {
  std::ifstream fm(o.load + "/meta.txt");
  if (!fm) { std::cerr << "no meta.txt in " << o.load << "\n"; return 3; }
  std::map<std::string, double> meta;
  std::string line;
  std::getline(fm, line);
  {
    std::istringstream is(line);
    std::string k;
    double v;
    while (is >> k >> v) meta[k] = v;
  }
  const int lx = (int)meta["lx"], ly = (int)meta["ly"], il = (int)meta["il"], ir = (int)meta["ir"];
  psize = o.threads;
  omp_set_num_threads(o.threads);
  std::streambuf* saved = std::cout.rdbuf();
  std::ostringstream sink;
  std::cout.rdbuf(sink.rdbuf());
  DMRG<S, Sym> chain(lx, ly, (int)meta["D"], 1, (int)meta["sec"], 0);
  std::cout.rdbuf(saved);
  Opts g = o;
  g.open = (int)meta["open"];
  g.J2 = meta["J2"];
  patch_geometry(chain, g);
  if constexpr (Sym::has_cgc) {
    // fac_hamilt_vec for 2J beyond the constructor's max_angm = 20, computed with the
    // reference's own Dense / CGCTable code by the formula of src/cgc_tables.cpp:153-164
    // table size: past the largest sector label of the problem's psi (+ the channel 2J = 2)
    int M = 64;
    {
      std::ifstream fp(o.load + "/psi.txt");
      std::string w;
      while (fp >> w)
        if (w == "q") {
          std::string x;
          while (fp >> x && x != "d") M = std::max(M, std::atoi(x.c_str()) + 8);
        }
    }
    double*** f = new double**[M];
    std::vector<Dense<double>> sg(M);
    Dense<double> c, t1, t2;
    for (int i = 0; i < M; ++i) sg[i].make_singlet(i);
    for (int i = 0; i < M; ++i) {
      f[i] = new double*[M];
      for (int j = 0; j < M; ++j) {
        f[i][j] = new double[M]();
        for (int k = 0; k < M; ++k)
          if (j <= 6 && k >= std::abs(i - j) && k <= i + j && (i % 2 == k % 2)) {
            c.make_cgc(i, j, k);
            t1.contract(c, 0, sg[i], 1);
            t2.contract(t1, 0, sg[j], 1);
            t1.contract(t2, 0, sg[k], 1);
            f[i][j][k] = c.inner_prod_u(t1) * std::sqrt((double)(j + 1));
          }
      }
    }
    g_cgc_tables->fac_hamilt_vec = f;  // the old 20^3 table is left allocated
  }
  BlockTensor<S, Sym> vec, out;
  bool ok = load_tensor(o.load, "psi", vec, true);
  load_tensor(o.load, "hh_il", chain.hh[il], false);
  load_tensor(o.load, "hh_ir", chain.hh[ir], false);
  for (int k = 0; k < chain.ns; ++k) {
    load_tensor(o.load, "opr_il_" + std::to_string(k), chain.opr[il][k], false);
    load_tensor(o.load, "opr_ir_" + std::to_string(k), chain.opr[ir][k], false);
  }
  if (!ok) { std::cerr << "no psi in " << o.load << "\n"; return 3; }
  std::cout.rdbuf(sink.rdbuf());
  chain.hamiltonian_vector_multiplication_idmrg(il, ir, vec, out);
  std::cout.rdbuf(saved);
  {
    // result in the block order of psi (missing blocks written as zeros)
    std::ofstream fo(o.load + "/hpsi_ref.bin", std::ios::binary);
    std::vector<int> angm(2), bdim(2);
    for (int i = 0; i < vec.nten; ++i) {
      if (vec.data_blocks[i].check_null()) continue;
      const long n = vec.data_blocks[i].get_nelem();
      if (i < out.nten && !out.data_blocks[i].check_null())
        fo.write(reinterpret_cast<const char*>(out.data_blocks[i].getptr()), sizeof(S) * n);
      else {
        std::vector<S> z(n, S(0));
        fo.write(reinterpret_cast<const char*>(z.data()), sizeof(S) * n);
      }
    }
  }
  const int reps = std::max(o.bench_heff, 1);
  std::cout.rdbuf(sink.rdbuf());
  auto a = std::chrono::steady_clock::now();
  for (int r = 0; r < reps; ++r) chain.hamiltonian_vector_multiplication_idmrg(il, ir, vec, out);
  auto b = std::chrono::steady_clock::now();
  std::cout.rdbuf(saved);
  std::cout << std::setprecision(10) << "BENCH_HEFF calls " << reps << " seconds "
            << std::chrono::duration<double>(b - a).count() << " threads " << o.threads << "\n";
  return 0;
}

int main(int argc, char** argv) {
  Opts o;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto nxt = [&]() { return std::string(argv[++i]); };
    if (a == "-sym") o.sym = nxt() == "su2" ? 1 : 0;
    else if (a == "-cplx") o.cplx = std::stoi(nxt());
    else if (a == "-lx") o.lx = std::stoi(nxt());
    else if (a == "-ly") o.ly = std::stoi(nxt());
    else if (a == "-L") { o.lx = 1; o.ly = std::stoi(nxt()); }
    else if (a == "-d") o.D = std::stoi(nxt());
    else if (a == "-sec") o.sec = std::stoi(nxt());
    else if (a == "-sweeps") o.sweeps = std::stoi(nxt());
    else if (a == "-threads") o.threads = std::stoi(nxt());
    else if (a == "-maxangm") o.maxangm = std::stoi(nxt());
    else if (a == "-open") o.open = std::stoi(nxt());
    else if (a == "-J2") o.J2 = std::stod(nxt());
    else if (a == "-dump") o.dump = nxt();
    else if (a == "-save") o.save = nxt();
    else if (a == "-read") o.read = nxt();
    else if (a == "-load") o.load = nxt();
    else if (a == "-bench_heff") o.bench_heff = std::stoi(nxt());
    else if (a == "-verbose") o.quiet = 0;
    else if (a == "-mlanc") o.mlanc = std::stoi(nxt());
    else if (a == "-lanc_check") o.lanc_check = std::stod(nxt());
    else if (a == "-sweepdir") o.sweepdir = nxt();
    else if (a == "-exci") o.exci = std::stoi(nxt());
    else { std::cerr << "unknown option " << a << "\n"; return 2; }
  }
  ref_lanczos_mlanc = o.mlanc;
  ref_lanczos_check = o.lanc_check;
  if (!o.load.empty()) {
    if (o.sym == 0 && o.cplx == 0) return run_load<double, U1Symmetry>(o);
    if (o.sym == 0 && o.cplx == 1) return run_load<dcmplex, U1Symmetry>(o);
    if (o.sym == 1 && o.cplx == 0) return run_load<double, SU2Symmetry>(o);
    return run_load<dcmplex, SU2Symmetry>(o);
  }
  if (o.sym == 0 && o.cplx == 0) return run<double, U1Symmetry>(o);
  if (o.sym == 0 && o.cplx == 1) return run<dcmplex, U1Symmetry>(o);
  if (o.sym == 1 && o.cplx == 0) return run<double, SU2Symmetry>(o);
  return run<dcmplex, SU2Symmetry>(o);
}
