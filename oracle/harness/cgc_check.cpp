// cgc_check.cpp -- test infrastructure: the library's SU(2) factors against the
// reference's own tables.
//
// The library computes each reduced-matrix factor on first use and memoises it
// (symmetry-adapted-dmrg-library_b200/csrc/cgc.cpp, sadmrg::CGCFactors); the
// reference fills dense tables up to an angular-momentum cutoff M
// (makeup_clebsch_gordan_coefficient_tensors, src/cgc_tables.cpp:102-357).  This
// program builds the reference's tables for one physical spin and cutoff and
// compares every entry -- zeros included -- with the library's factor for the
// same tuple:
//   fac_hamilt_vec[i][j][k]                              hamilt_vec(i, j, k)
//   fac_operator_onsite_{left,rght}[j][m][l][i][p0+p1*P2]    onsite(0/1, j, m, l, i, p0, p1)
//   fac_operator_transformation_{left,rght}[j][m][l][i][k][p0]  transformation(0/1, j, m, l, i, k, p0)
//   fac_operator_pairup_{left,rght}[j][i][k][m][p0+p1*P2]    pairup(0/1, j, i, k, m, p0, p1)
//
// usage: cgc_check <physpn (2S)> <max_angm>
// prints one line per table: name, entries, nonzero entries, largest |difference|,
// entries off by more than 1e-12 (relative to max(1, |value|)); exits 1 on any.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <sstream>

#include "cgc_tables.hpp"
#include "../../symmetry-adapted-dmrg-library_b200/csrc/cgc.hpp"

namespace {

struct Tally {
  const char* name;
  long entries = 0, nonzero = 0, bad = 0;
  double maxdiff = 0.0;
  void add(double ref, double got) {
    ++entries;
    if (ref != 0.0) ++nonzero;
    const double d = std::fabs(ref - got);
    if (d > maxdiff) maxdiff = d;
    if (d > 1e-12 * std::fmax(1.0, std::fabs(ref))) ++bad;
  }
  void print() const {
    std::printf("%s entries %ld nonzero %ld maxdiff %.3e mismatches %ld\n", name, entries, nonzero, maxdiff, bad);
  }
};

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: cgc_check <physpn> <max_angm>\n");
    return 2;
  }
  const int physpn = std::atoi(argv[1]), M = std::atoi(argv[2]);
  if (physpn < 1 || physpn > 4 || M < 7 || M > 24) {
    std::fprintf(stderr, "cgc_check: physpn 1..4, max_angm 7..24\n");
    return 2;
  }
  CGCTables t;
  {
    // the reference reports progress on stdout; keep this program's output to the tallies
    std::ostringstream sink;
    std::streambuf* old = std::cout.rdbuf(sink.rdbuf());
    makeup_clebsch_gordan_coefficient_tensors(physpn, M, t);
    std::cout.rdbuf(old);
  }
  sadmrg::CGCFactors f(physpn);
  const int P2 = 2 * physpn + 1;

  Tally hv{"hamilt_vec"};
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < M; ++j)
      for (int k = 0; k < M; ++k) hv.add(t.fac_hamilt_vec[i][j][k], f.hamilt_vec(i, j, k));

  Tally on[2] = {{"onsite_left"}, {"onsite_rght"}};
  Tally tr[2] = {{"transformation_left"}, {"transformation_rght"}};
  Tally pu[2] = {{"pairup_left"}, {"pairup_rght"}};
  for (int flag = 0; flag < 2; ++flag) {
    double***** ons = flag ? t.fac_operator_onsite_rght : t.fac_operator_onsite_left;
    double****** trs = flag ? t.fac_operator_transformation_rght : t.fac_operator_transformation_left;
    double***** pus = flag ? t.fac_operator_pairup_rght : t.fac_operator_pairup_left;
    for (int a = 0; a < M; ++a)
      for (int b = 0; b < M; ++b)
        for (int c = 0; c < M; ++c)
          for (int d = 0; d < M; ++d) {
            for (int p1 = 0; p1 < P2; ++p1)
              for (int p0 = 0; p0 < P2; ++p0) {
                // onsite: [j = a][m = b][l = c][i = d]; pairup: [j = a][i = b][k = c][m = d]
                on[flag].add(ons[a][b][c][d][p0 + p1 * P2], f.onsite(flag, a, b, c, d, p0, p1));
                pu[flag].add(pus[a][b][c][d][p0 + p1 * P2], f.pairup(flag, a, b, c, d, p0, p1));
              }
            // transformation: [j = a][m = b][l = c][i = d][k][p0]
            for (int k = 0; k < M; ++k)
              for (int p0 = 0; p0 < P2; ++p0)
                tr[flag].add(trs[a][b][c][d][k][p0], f.transformation(flag, a, b, c, d, k, p0));
          }
  }
  long bad = hv.bad;
  hv.print();
  for (int flag = 0; flag < 2; ++flag) {
    on[flag].print();
    tr[flag].print();
    pu[flag].print();
    bad += on[flag].bad + tr[flag].bad + pu[flag].bad;
  }
  return bad ? 1 : 0;
}
