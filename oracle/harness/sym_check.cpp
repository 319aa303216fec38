// sym_check.cpp -- test infrastructure: the library's sector bookkeeping against
// the reference's, on seeded random bonds.
//
// The library restates the reference's U(1) / SU(2) conventions in one header
// (symmetry-adapted-dmrg-library_b200/csrc/symmetry.hpp: Bond::set, Bond::fuse,
// Struct::block, Struct::index, Struct::allowed_labels).  This program draws
// random bonds and tensor structures and compares, for each symmetry:
//   fuse of two bonds: direction, sector labels (order included) and dims
//     vs U1Bond::fuse / SU2Bond::fuse (src/symmetry/u1.cpp, su2.cpp);
//   every block index of a 2-4 bond structure: allowed or not, labels and dims
//     vs U1Struct / SU2Struct::get_tensor_argument, and the block index found
//     back from the labels vs get_tensor_index;
//   the cyclic move of a bond (Struct::shifted vs the reference's shift, every
//     (i0, i1) pair of the structure): each bond's direction, labels and dims.
//
// usage: sym_check <cases> <seed>
// prints one line per symmetry (cases, blocks, allowed blocks, mismatches, shifts);
// exits 1 on any mismatch.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "symmetry/su2.hpp"
#include "symmetry/u1.hpp"
#include "../../symmetry-adapted-dmrg-library_b200/csrc/symmetry.hpp"

namespace {

std::mt19937 rng;

int rnd(int lo, int hi) { return std::uniform_int_distribution<int>(lo, hi)(rng); }

// distinct labels in [lo, hi], random order; dims in [1, 5]
void draw(int n, int lo, int hi, std::vector<int>& q, std::vector<int>& d) {
  std::vector<int> pool;
  for (int x = lo; x <= hi; ++x) pool.push_back(x);
  std::shuffle(pool.begin(), pool.end(), rng);
  q.assign(pool.begin(), pool.begin() + n);
  d.resize(n);
  for (int& x : d) x = rnd(1, 5);
}

template <class RB>
bool same_bond(const RB& r, const sadmrg::Bond& b) {
  if (r.get_bonddir() != b.dir || r.get_nmoment() != b.nmom()) return false;
  for (int i = 0; i < b.nmom(); ++i)
    if (r.get_angularmoment(i) != b.q[i] || r.get_bonddim(i) != b.d[i]) return false;
  return true;
}

struct Tally {
  const char* name;
  long cases = 0, blocks = 0, allowed = 0, shifts = 0, bad = 0;
};

template <class RB, class RS>
void run(Tally& t, sadmrg::Sym sym, int cases) {
  const bool su2 = sym == sadmrg::Sym::SU2;
  for (int c = 0; c < cases; ++c) {
    ++t.cases;
    // fuse
    {
      std::vector<int> q1, d1, q2, d2;
      draw(rnd(1, 4), su2 ? 0 : -4, su2 ? 6 : 4, q1, d1);
      draw(rnd(1, 4), su2 ? 0 : -4, su2 ? 6 : 4, q2, d2);
      const int dir1 = rnd(0, 1) ? 1 : -1;
      const int dir2 = su2 ? dir1 : (rnd(0, 1) ? 1 : -1);
      RB a, b, f;
      a.set(dir1, (int)q1.size(), q1.data(), d1.data());
      b.set(dir2, (int)q2.size(), q2.data(), d2.data());
      f.fuse(a, b);
      const sadmrg::Bond la(dir1, q1, d1), lb(dir2, q2, d2);
      if (!same_bond(a, la) || !same_bond(b, lb) || !same_bond(f, sadmrg::Bond::fuse(sym, la, lb))) ++t.bad;
    }
    // block enumeration of a structure
    const int nb = rnd(2, 4);
    std::vector<RB> rb(nb);
    std::vector<sadmrg::Bond> lb;
    for (int k = 0; k < nb; ++k) {
      std::vector<int> q, d;
      draw(rnd(1, 4), su2 ? 0 : -3, su2 ? 5 : 3, q, d);
      const int dir = rnd(0, 1) ? 1 : -1;
      rb[k].set(dir, (int)q.size(), q.data(), d.data());
      lb.emplace_back(dir, q, d);
    }
    const int locspin = su2 ? rnd(0, 3) : rnd(-3, 3);
    RS rs;
    rs.set_struct(nb, locspin, rb.data());
    const sadmrg::Struct ls(sym, locspin, lb);
    if (rs.get_nten() != ls.nten()) { ++t.bad; continue; }
    for (int i0 = 0; i0 < nb; ++i0)
      for (int i1 = 0; i1 < nb; ++i1) {
        ++t.shifts;
        RS r2;
        r2.set_struct(nb, locspin, rb.data());
        r2.shift(i0, i1);
        const sadmrg::Struct l2 = ls.shifted(i0, i1);
        bool ok = r2.get_nbond() == l2.nbond();
        for (int k = 0; ok && k < nb; ++k) {
          RB got;
          r2.get_bond(k, got);
          ok = same_bond(got, l2.bonds[k]);
        }
        if (!ok) ++t.bad;
      }
    for (long i = 0; i < ls.nten(); ++i) {
      ++t.blocks;
      int rq[8], rd[8], q[8], d[8];
      const bool ra = rs.get_tensor_argument((int)i, rq, rd);
      const bool la2 = ls.block(i, q, d);
      bool ok = ra == la2;
      for (int k = 0; ok && k < nb; ++k) ok = rq[k] == q[k] && rd[k] == d[k];
      if (ok && la2) {
        ++t.allowed;
        ok = rs.get_tensor_index(q) == (int)i && ls.index(q) == i;
      }
      if (!ok) ++t.bad;
    }
  }
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: sym_check <cases> <seed>\n");
    return 2;
  }
  const int cases = std::atoi(argv[1]);
  rng.seed((unsigned)std::atoi(argv[2]));
  Tally u{"u1"}, s{"su2"};
  run<U1Bond, U1Struct>(u, sadmrg::Sym::U1, cases);
  run<SU2Bond, SU2Struct>(s, sadmrg::Sym::SU2, cases);
  for (const Tally* t : {&u, &s})
    std::printf("%s cases %ld blocks %ld allowed %ld mismatches %ld shifts %ld\n", t->name, t->cases, t->blocks,
                t->allowed, t->bad, t->shifts);
  return (u.bad || s.bad) ? 1 : 0;
}
