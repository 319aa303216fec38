// cgc.cpp -- SU(2) Clebsch-Gordan coefficients and memoised reduced-matrix factors.
#include "cgc.hpp"

#include <cmath>
#include <cstdlib>

#include "common.hpp"

namespace sadmrg {

static double fact(int n) {
  double f = 1.0;
  for (int i = 2; i <= n; ++i) f *= i;
  return f;
}

// Racah's closed form; all labels doubled (2J, 2M).
double clebsch_gordan(int j1, int m1, int j2, int m2, int j3, int m3) {
  if (m1 + m2 != m3) return 0.0;
  if (j3 < std::abs(j1 - j2) || j3 > j1 + j2) return 0.0;
  if ((j1 + j2 + j3) % 2 != 0) return 0.0;
  const double pre = std::sqrt((double)(j3 + 1) * fact((j3 + j1 - j2) / 2) * fact((j3 - j1 + j2) / 2) *
                               fact((j1 + j2 - j3) / 2) / fact((j1 + j2 + j3) / 2 + 1));
  const double mf = std::sqrt(fact((j1 + m1) / 2) * fact((j1 - m1) / 2) * fact((j2 + m2) / 2) *
                              fact((j2 - m2) / 2) * fact((j3 + m3) / 2) * fact((j3 - m3) / 2));
  const int a = (j1 + j2 - j3) / 2, b = (j1 - m1) / 2, c = (j2 + m2) / 2;
  const int dd = (j3 - j2 + m1) / 2, e = (j3 - j1 - m2) / 2;
  double s = 0.0;
  for (int t = 0; t <= (j1 + j2 + j3) / 2; ++t) {
    if (a - t < 0 || b - t < 0 || c - t < 0 || dd + t < 0 || e + t < 0) continue;
    const double den = fact(t) * fact(a - t) * fact(b - t) * fact(c - t) * fact(dd + t) * fact(e + t);
    s += ((t % 2) ? -1.0 : 1.0) / den;
  }
  return pre * mf * s;
}

void HDense::alloc(std::vector<int> d) {
  dims = std::move(d);
  long n = 1;
  for (int x : dims) n *= x;
  v.assign(n, 0.0);
}

void HDense::make_cgc(int j1, int j2, int j3) {
  alloc({j1 + 1, j2 + 1, j3 + 1});
  for (int i = 0; i <= j1; ++i)
    for (int j = 0; j <= j2; ++j)
      for (int k = 0; k <= j3; ++k)
        v[i + j * (j1 + 1) + k * (j1 + 1) * (j2 + 1)] =
            clebsch_gordan(j1, 2 * i - j1, j2, 2 * j - j2, j3, 2 * k - j3);
}

void HDense::make_singlet(int jj) {
  alloc({jj + 1, jj + 1});
  for (int i = 0; i <= jj; ++i)
    for (int j = 0; j <= jj; ++j) {
      int m1 = 2 * i - jj, m2 = 2 * j - jj;
      if (m1 + m2 == 0) v[i + j * (jj + 1)] = ((((jj - m1) / 2) % 2) == 0 ? 1.0 : -1.0) / std::sqrt((double)(jj + 1));
    }
}

void HDense::make_identity(int jj) {
  alloc({jj + 1, jj + 1});
  for (int i = 0; i <= jj; ++i) v[i + i * (jj + 1)] = 1.0;
}

void HDense::shift(int i0, int i1) {
  if (i0 == i1) return;
  const int n = nbond();
  const int ish = (i1 > i0) ? (i1 - i0) : (n - (i0 - i1));
  std::vector<int> nd(n);
  for (int i = 0; i < n; ++i) nd[(i + ish) % n] = dims[i];
  const int p = n - ish;
  long B = 1, A = 1;
  for (int i = 0; i < p; ++i) B *= dims[i];
  for (int i = p; i < n; ++i) A *= dims[i];
  std::vector<double> t(v.size());
  for (long b = 0; b < B; ++b)
    for (long a = 0; a < A; ++a) t[a + A * b] = v[b + B * a];
  v.swap(t);
  dims = nd;
}

void HDense::exchangeindex(int i1, int i2) {
  if (i1 == i2) return;
  if (i1 > i2) std::swap(i1, i2);
  long A = 1, C = 1, E = 1;
  const long Bd = dims[i1], Dd = dims[i2];
  for (int i = 0; i < i1; ++i) A *= dims[i];
  for (int i = i1 + 1; i < i2; ++i) C *= dims[i];
  for (int i = i2 + 1; i < nbond(); ++i) E *= dims[i];
  std::vector<double> t(v.size());
  for (long e = 0; e < E; ++e)
    for (long d = 0; d < Dd; ++d)
      for (long c = 0; c < C; ++c)
        for (long b = 0; b < Bd; ++b) {
          const long src = A * (b + Bd * (c + C * (d + Dd * e)));
          const long dst = A * (d + Dd * (c + C * (b + Bd * e)));
          for (long a = 0; a < A; ++a) t[dst + a] = v[src + a];
        }
  v.swap(t);
  std::swap(dims[i1], dims[i2]);
}

void HDense::mergeindex(int i0, int i1) {
  SADMRG_REQUIRE(i1 == i0 + 1, SADMRG_ERR_ARG, "mergeindex: indices not adjacent");
  dims[i0] *= dims[i1];
  dims.erase(dims.begin() + i1);
}

void HDense::separateindex(int i, int d0, int d1) {
  SADMRG_REQUIRE(d0 * d1 == dims[i], SADMRG_ERR_ARG, "separateindex: inconsistent dims");
  dims[i] = d0;
  dims.insert(dims.begin() + i + 1, d1);
}

double HDense::inner_prod_u(const HDense& o) const {
  double s = 0.0;
  for (long i = 0; i < nelem(); ++i) s += v[i] * o.v[i];
  return s;
}

bool HDense::is_zero() const {
  for (double x : v)
    if (std::fabs(x) > 1e-12) return false;
  return true;
}

bool HDense::proportional_to(const HDense& o, double& ratio) const {
  ratio = 0.0;
  if (nelem() != o.nelem() || dims != o.dims) return false;
  if (is_zero()) return true;
  long pos = 0;
  double mx = 0.0;
  for (long i = 0; i < o.nelem(); ++i)
    if (std::fabs(o.v[i]) > mx) { mx = std::fabs(o.v[i]); pos = i; }
  if (mx <= 1e-12) return false;
  ratio = v[pos] / o.v[pos];
  for (long i = 0; i < nelem(); ++i) {
    const bool za = std::fabs(v[i]) <= 1e-12, zb = std::fabs(o.v[i]) <= 1e-12;
    if (za && zb) continue;
    if (za != zb) return false;
    if (std::fabs(v[i] / o.v[i] - ratio) > 1e-12) return false;
  }
  return true;
}

void HDense::contract(const HDense& A, int ia, const HDense& B, int ib) {
  SADMRG_REQUIRE(A.dims[ia] == B.dims[ib], SADMRG_ERR_ARG, "HDense::contract: dims mismatch");
  HDense a = A, b = B;
  a.shift(ia, A.nbond() - 1);  // contracted bond last, rest in cyclic order from ia+1
  b.shift(ib, 0);              // contracted bond first, rest in cyclic order from ib+1
  const long k = A.dims[ia];
  const long m = A.nelem() / k, n = B.nelem() / k;
  std::vector<int> nd;
  for (int i = 0; i < A.nbond() - 1; ++i) nd.push_back(A.dims[(ia + 1 + i) % A.nbond()]);
  for (int i = 0; i < B.nbond() - 1; ++i) nd.push_back(B.dims[(ib + 1 + i) % B.nbond()]);
  std::vector<double> r(m * n, 0.0);
  for (long c = 0; c < n; ++c)
    for (long kk = 0; kk < k; ++kk) {
      const double bv = b.v[kk + k * c];
      if (bv == 0.0) continue;
      for (long rr = 0; rr < m; ++rr) r[rr + m * c] += a.v[rr + m * kk] * bv;
    }
  dims = nd;
  v.swap(r);
}

void HDense::overlap_initial(const HDense& t1, const HDense& t2) {
  const long k = (long)t1.dims[0] * t1.dims[1];
  const long m = t1.nelem() / k, n = t2.nelem() / k;
  std::vector<double> r(m * n, 0.0);
  for (long c = 0; c < n; ++c)
    for (long rr = 0; rr < m; ++rr) {
      double s = 0.0;
      for (long kk = 0; kk < k; ++kk) s += t1.v[kk + k * rr] * t2.v[kk + k * c];
      r[rr + m * c] = s;
    }
  dims = {t1.dims[2], t2.dims[2]};
  v.swap(r);
}

void HDense::operator_initial(const HDense& t1, const HDense& t2, const HDense& t3, int flag) {
  if (t3.dims[0] == 1 && t3.dims[1] == 1 && t3.dims[2] == 1) {
    overlap_initial(t1, t2);
    scale(t3.v[0]);
    separateindex(0, dims[0], 1);
    return;
  }
  HDense a, b = t2;
  if (flag == 0) {
    a.contract(t1, 1, t3, 0);
    a.exchangeindex(1, 2);
    a.mergeindex(2, 3);
    b.mergeindex(0, 1);
    contract(a, 2, b, 0);
  } else {
    a.contract(t1, 0, t3, 0);
    a.shift(3, 0);
    a.mergeindex(0, 1);
    b.mergeindex(0, 1);
    contract(a, 0, b, 0);
  }
}

void HDense::operator_transformation(const HDense& t1, const HDense& t2, const HDense& t3, int flag) {
  if (t3.dims[1] == 1 && ((flag == 0 && t1.dims[1] == 1) || (flag == 1 && t1.dims[0] == 1))) {
    const long k1 = t3.dims[0], m1 = t1.nelem() / k1, n1 = t3.nelem() / k1;
    std::vector<double> T(m1 * n1, 0.0);
    for (long c = 0; c < n1; ++c)
      for (long r = 0; r < m1; ++r) {
        double s = 0.0;
        for (long kk = 0; kk < k1; ++kk) s += t1.v[kk + k1 * r] * t3.v[kk + k1 * c];
        T[r + m1 * c] = s;
      }
    const long k2 = t3.dims[2], m2 = (m1 * n1) / k2, n2 = t2.nelem() / k2;
    std::vector<double> R(m2 * n2, 0.0);
    for (long c = 0; c < n2; ++c)
      for (long kk = 0; kk < k2; ++kk)
        for (long r = 0; r < m2; ++r) R[r + m2 * c] += T[r + m2 * kk] * t2.v[kk + k2 * c];
    dims = {t1.dims[2], t3.dims[1], t2.dims[2]};
    v.swap(R);
    return;
  }
  HDense a, b = t2;
  if (flag == 0) {
    a.contract(t1, 0, t3, 0);
    a.shift(1, 0);
  } else {
    a.contract(t1, 1, t3, 0);
    a.exchangeindex(1, 2);
  }
  a.mergeindex(2, 3);
  b.mergeindex(0, 1);
  contract(a, 2, b, 0);
}

void HDense::operator_pairup(const HDense& uu, const HDense& vv, const HDense& op1, const HDense& op2, int flag) {
  if (op1.dims[1] == 1 && op2.dims[0] == 1 && op2.dims[1] == 1 && op2.dims[2] == 1) {
    operator_transformation(uu, vv, op1, flag);
    mergeindex(0, 1);
    scale(op2.v[0]);
    return;
  }
  HDense a, b = op2, c, w = vv;
  b.mergeindex(0, 1);
  w.mergeindex(0, 1);
  if (flag == 0) {
    a.contract(uu, 0, op1, 0);
    a.exchangeindex(1, 2);
    a.mergeindex(0, 1);
    c.contract(a, 0, b, 0);
    c.mergeindex(1, 2);
    contract(c, 1, w, 0);
  } else {
    a.contract(uu, 1, op1, 0);
    a.shift(1, 0);
    a.mergeindex(0, 1);
    c.contract(b, 0, a, 0);
    c.mergeindex(0, 1);
    contract(c, 0, w, 0);
  }
}

uint64_t CGCFactors::key(int kind, int a, int b, int c, int d, int e, int f, int g) {
  auto u = [](int x) { return (uint64_t)(x & 0x1ff); };
  return (u(kind) << 54) | (u(a) << 45) | (u(b) << 36) | (u(c) << 27) | (u(d) << 18) | (u(e) << 9) | u(f) |
         ((uint64_t)(g & 0x1) << 63);
}

static inline bool tri(int a, int b, int c) { return c >= std::abs(a - b) && c <= a + b; }
static inline bool chan_ok(int m) { return m >= 0 && m <= 6 && (m % 2) == 0; }

double CGCFactors::hamilt_vec(int i, int j, int k) {
  if (!(tri(i, j, k) && (i % 2 == k % 2))) return 0.0;
  const uint64_t kk = key(1, i, j, k, 0, 0, 0, 0);
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = memo_.find(kk);
    if (it != memo_.end()) return it->second;
  }
  HDense C, si, sj, sk, t1, t2;
  C.make_cgc(i, j, k);
  si.make_singlet(i);
  sj.make_singlet(j);
  sk.make_singlet(k);
  t1.contract(C, 0, si, 1);
  t2.contract(t1, 0, sj, 1);
  t1.contract(t2, 0, sk, 1);
  const double r = C.inner_prod_u(t1) * std::sqrt((double)(j + 1));
  std::lock_guard<std::mutex> g(mu_);
  memo_[kk] = r;
  return r;
}

double CGCFactors::onsite(int flag, int j, int m, int l, int i, int p0, int p1) {
  if (p0 < 0 || p1 < 0 || p0 >= p2_ || p1 >= p2_ || !chan_ok(m)) return 0.0;
  if (!(tri(i, p0, j) && tri(i, p1, l) && tri(j, m, l) && (j % 2 == l % 2) && tri(p0, m, p1))) return 0.0;
  const uint64_t kk = key(2, j, m, l, i, p0, p1, flag);
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = memo_.find(kk);
    if (it != memo_.end()) return it->second;
  }
  HDense a, b, c, r, s;
  if (flag == 0) { a.make_cgc(i, p0, j); b.make_cgc(i, p1, l); }
  else           { a.make_cgc(p0, i, j); b.make_cgc(p1, i, l); }
  c.make_cgc(p0, m, p1);
  r.operator_initial(a, b, c, flag);
  s.make_cgc(j, m, l);
  double ratio = 0.0;
  r.proportional_to(s, ratio);
  std::lock_guard<std::mutex> g(mu_);
  memo_[kk] = ratio;
  return ratio;
}

double CGCFactors::transformation(int flag, int j, int m, int l, int i, int k, int p0) {
  if (p0 < 0 || p0 >= p2_ || !chan_ok(m)) return 0.0;
  if (!(tri(i, p0, j) && tri(k, p0, l) && tri(i, m, k) && (k % 2 == i % 2) && tri(j, m, l) && (j % 2 == l % 2)))
    return 0.0;
  const uint64_t kk = key(3, j, m, l, i, k, p0, flag);
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = memo_.find(kk);
    if (it != memo_.end()) return it->second;
  }
  HDense a, b, c, r, s;
  if (flag == 0) { a.make_cgc(i, p0, j); b.make_cgc(k, p0, l); }
  else           { a.make_cgc(p0, i, j); b.make_cgc(p0, k, l); }
  c.make_cgc(i, m, k);
  r.operator_transformation(a, b, c, flag);
  s.make_cgc(j, m, l);
  double ratio = 0.0;
  r.proportional_to(s, ratio);
  std::lock_guard<std::mutex> g(mu_);
  memo_[kk] = ratio;
  return ratio;
}

double CGCFactors::pairup(int flag, int j, int i, int k, int m, int p0, int p1) {
  if (p0 < 0 || p1 < 0 || p0 >= p2_ || p1 >= p2_ || !chan_ok(m)) return 0.0;
  if (!(tri(i, p0, j) && tri(k, p1, j) && tri(i, m, k) && tri(p0, m, p1))) return 0.0;
  const uint64_t kk = key(4, j, i, k, m, p0, p1, flag);
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = memo_.find(kk);
    if (it != memo_.end()) return it->second;
  }
  HDense t, sm, a, b, c, r, id;
  HDense base;
  base.make_cgc(p0, m, p1);
  sm.make_singlet(m);
  t.contract(base, 1, sm, 1);
  t.shift(0, 2);
  t.scale(std::sqrt((double)(m + 1)));
  if (flag == 0) { a.make_cgc(i, p0, j); b.make_cgc(k, p1, j); }
  else           { a.make_cgc(p0, i, j); b.make_cgc(p1, k, j); }
  c.make_cgc(i, m, k);
  r.operator_pairup(a, b, c, t, flag);
  id.make_identity(j);
  double ratio = 0.0;
  r.proportional_to(id, ratio);
  std::lock_guard<std::mutex> g(mu_);
  memo_[kk] = ratio;
  return ratio;
}

}  // namespace sadmrg
