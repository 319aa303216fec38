// symmetry.hpp -- sector bookkeeping for U(1) charges and SU(2) multiplets.
//
// Host-only integer metadata.  The conventions (sector order, fusion rules,
// block enumeration, allowed-block test) follow the reference exactly, because
// the block order of every tensor, and therefore every task list and every
// checkpoint file, depends on them:
//   Bond::set sorts sectors ascending          symmetry/u1.cpp:19-27, su2.cpp:22-29
//   U(1) fuse (charges add, dir = -dir2)        src/symmetry/u1.cpp:111-141,144-167
//   SU(2) fuse (triangle rule, dir = -dir1)     src/symmetry/su2.cpp:182-254
//   block index = mixed radix, bond 0 fastest   src/symmetry/u1.cpp:322-339, su2.cpp:432-449
//   allowed: U(1) sum dir*q == locspin          src/symmetry/u1.cpp:348-378
//            SU(2) triangle reachability        src/symmetry/su2.cpp:483-507
#pragma once
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "common.hpp"

namespace sadmrg {

enum class Sym : int { U1 = 0, SU2 = 1 };

struct Bond {
  int dir = 0;
  std::vector<int> q;  // charge (U1) or 2J (SU2), ascending
  std::vector<int> d;  // reduced dimension per sector

  Bond() = default;
  Bond(int dir_, std::vector<int> q_, std::vector<int> d_) { set(dir_, std::move(q_), std::move(d_)); }

  void set(int dir_, std::vector<int> q_, std::vector<int> d_) {
    dir = dir_;
    q = std::move(q_);
    d = std::move(d_);
    // the reference's exchange sort (ascending by sector label)
    int n = (int)q.size();
    for (int i = 0; i < n - 1; ++i)
      for (int j = i + 1; j < n; ++j)
        if (q[j] < q[i]) { std::swap(q[i], q[j]); std::swap(d[i], d[j]); }
  }
  int nmom() const { return (int)q.size(); }
  int index_of(int qq) const {
    for (int i = 0; i < nmom(); ++i)
      if (q[i] == qq) return i;
    return -1;
  }
  void invert() { dir = -dir; }
  bool operator==(const Bond& o) const { return dir == o.dir && q == o.q && d == o.d; }
  bool operator!=(const Bond& o) const { return !(*this == o); }
  int total_dim(Sym s) const {
    int t = 0;
    for (int i = 0; i < nmom(); ++i) t += d[i] * (s == Sym::SU2 ? q[i] + 1 : 1);
    return t;
  }

  // fuse two bonds (reference semantics, including the output direction)
  static Bond fuse(Sym s, const Bond& b1, const Bond& b2) {
    std::vector<int> val, dim;
    auto add = [&](int c, int dd) {
      for (size_t k = 0; k < val.size(); ++k)
        if (val[k] == c) { dim[k] += dd; return; }
      val.push_back(c);
      dim.push_back(dd);
    };
    if (s == Sym::U1) {
      for (int j = 0; j < b2.nmom(); ++j)
        for (int i = 0; i < b1.nmom(); ++i) {
          int c = (b1.dir * b2.dir == 1) ? b1.q[i] + b2.q[j] : -b1.q[i] + b2.q[j];
          add(c, b1.d[i] * b2.d[j]);
        }
      return Bond(-b2.dir, val, dim);
    }
    SADMRG_REQUIRE(b1.dir == b2.dir, SADMRG_ERR_ARG, "SU2 fuse: bond directions differ");
    for (int i = 0; i < b1.nmom(); ++i)
      for (int j = 0; j < b2.nmom(); ++j)
        for (int jk = std::abs(b1.q[i] - b2.q[j]); jk <= b1.q[i] + b2.q[j]; jk += 2)
          add(jk, b1.d[i] * b2.d[j]);
    return Bond(-b1.dir, val, dim);
  }
};

struct Struct {
  Sym sym = Sym::U1;
  int locspin = 0;
  std::vector<Bond> bonds;

  Struct() = default;
  Struct(Sym s, int ls, std::vector<Bond> b) : sym(s), locspin(ls), bonds(std::move(b)) {}

  int nbond() const { return (int)bonds.size(); }
  long nten() const {
    if (bonds.empty()) return 0;
    long n = 1;
    for (auto& b : bonds) n *= b.nmom();
    return n;
  }
  // decode block index -> per-bond sector indices
  void sectors(long i0, int* sec) const {
    for (int b = 0; b < nbond(); ++b) {
      sec[b] = (int)(i0 % bonds[b].nmom());
      i0 /= bonds[b].nmom();
    }
  }
  // labels and reduced dims of a block; returns whether the block is allowed
  bool block(long i0, int* q, int* d) const {
    int sec[8];
    sectors(i0, sec);
    for (int b = 0; b < nbond(); ++b) {
      q[b] = bonds[b].q[sec[b]];
      d[b] = bonds[b].d[sec[b]];
    }
    return allowed_labels(q);
  }
  // the reference's check_angularmoments
  bool allowed_labels(const int* q) const {
    int nb = nbond();
    if (nb <= 0) return false;
    if (sym == Sym::U1) {
      int tot = 0;
      for (int b = 0; b < nb; ++b) {
        if (bonds[b].index_of(q[b]) < 0) return false;
        tot += bonds[b].dir * q[b];
      }
      return tot == locspin;
    }
    if (nb == 1) return q[0] == locspin;
    int maxJ = 0;
    for (int b = 0; b < nb; ++b) maxJ += q[b];
    std::vector<unsigned char> reach(maxJ + 1, 0), next(maxJ + 1, 0);
    reach[q[0]] = 1;
    for (int b = 1; b < nb; ++b) {
      std::fill(next.begin(), next.end(), 0);
      for (int J = 0; J <= maxJ; ++J) {
        if (!reach[J]) continue;
        for (int K = std::abs(J - q[b]); K <= J + q[b]; K += 2) next[K] = 1;
      }
      reach.swap(next);
    }
    return (locspin >= 0 && locspin <= maxJ) ? reach[locspin] != 0 : false;
  }
  // block index from labels; -1 if a label is absent
  long index(const int* q) const {
    long i0 = 0;
    for (int b = nbond() - 1; b >= 0; --b) {
      int k = bonds[b].index_of(q[b]);
      if (k < 0) return -1;
      i0 = i0 * bonds[b].nmom() + k;
    }
    return i0;
  }
  long block_elems(long i0) const {
    int sec[8];
    sectors(i0, sec);
    long n = 1;
    for (int b = 0; b < nbond(); ++b) n *= bonds[b].d[sec[b]];
    return n;
  }
  // cyclic move of bond i0 to position i1 (reference shift semantics)
  Struct shifted(int i0, int i1) const {
    if (i0 == i1) return *this;
    int nb = nbond();
    int ish = (i1 > i0) ? (i1 - i0) : (nb - (i0 - i1));
    Struct s = *this;
    for (int i = 0; i < nb; ++i) s.bonds[(i + ish) % nb] = bonds[i];
    return s;
  }
  bool operator==(const Struct& o) const {
    return sym == o.sym && locspin == o.locspin && bonds == o.bonds;
  }
};

}  // namespace sadmrg
