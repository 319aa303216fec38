// cgc.hpp -- SU(2) Clebsch-Gordan coefficients and the reduced-matrix factors.
//
// The reference precomputes dense factor tables fac_*[M]^k for every 2J up to
// max_angm (src/cgc_tables.cpp:102-451): the transformation tables alone hold
// 2*M^5*P2 doubles (about 12 GB at M = 40) and any sector with 2J >= M reads
// out of bounds.  Here each factor is computed on first use, by the same
// contraction of explicit CGC tensors the reference uses, and memoised; so
// only the tuples a run touches are ever built and there is no 2J ceiling.
#pragma once
#include <cstdint>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace sadmrg {

// Small host dense tensor, column-major with index 0 fastest (reference layout,
// src/dense_inst.cpp:28-45).  Only the operations the CGC factors need.
struct HDense {
  std::vector<int> dims;
  std::vector<double> v;

  int nbond() const { return (int)dims.size(); }
  long nelem() const { return (long)v.size(); }
  void alloc(std::vector<int> d);
  bool null() const { return dims.empty() || v.empty(); }

  void make_cgc(int j1, int j2, int j3);
  void make_singlet(int jj);
  void make_identity(int jj);

  void shift(int i0, int i1);
  void exchangeindex(int i0, int i1);
  void mergeindex(int i0, int i1);
  void separateindex(int i, int d0, int d1);
  void scale(double s) { for (auto& x : v) x *= s; }
  double inner_prod_u(const HDense& o) const;
  bool is_zero() const;
  // ratio = this[pos] / o[pos] at the first largest |o| (Dense::is_proportional_to)
  bool proportional_to(const HDense& o, double& ratio) const;

  // *this = A contracted on A's bond ia with B's bond ib (Dense::contract)
  void contract(const HDense& A, int ia, const HDense& B, int ib);
  void overlap_initial(const HDense& t1, const HDense& t2);
  void operator_initial(const HDense& t1, const HDense& t2, const HDense& t3, int flag);
  void operator_transformation(const HDense& t1, const HDense& t2, const HDense& t3, int flag);
  void operator_pairup(const HDense& uu, const HDense& vv, const HDense& op1, const HDense& op2, int flag);
};

// Racah closed form for <j1 m1; j2 m2 | j3 m3>, every argument in 2J / 2M units.
double clebsch_gordan(int j1, int m1, int j2, int m2, int j3, int m3);

// Memoised factors.  Index order and skip conditions are the reference's
// (src/cgc_tables.cpp:146-357); a tuple outside the reference's loop bounds
// gives 0, exactly like an untouched table entry.
class CGCFactors {
 public:
  explicit CGCFactors(int physpn) : physpn_(physpn), p2_(2 * physpn + 1) {}
  int physpn() const { return physpn_; }
  int physpn2() const { return p2_; }

  double hamilt_vec(int i, int j, int k);
  double onsite(int flag, int j, int m, int l, int i, int p0, int p1);
  double transformation(int flag, int j, int m, int l, int i, int k, int p0);
  double pairup(int flag, int j, int i, int k, int m, int p0, int p1);

 private:
  int physpn_, p2_;
  std::mutex mu_;
  std::unordered_map<uint64_t, double> memo_;
  static uint64_t key(int kind, int a, int b, int c, int d, int e, int f, int g);
};

}  // namespace sadmrg
