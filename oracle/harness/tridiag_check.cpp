// tridiag_check.cpp -- test infrastructure: the library's tridiagonal eigensolver
// against the LAPACK routine the reference calls.
//
// The reference diagonalises each Lanczos tridiagonal with LAPACK dstev
// (Lanczos::diatridiag, src/dmrg_inst.cpp:1214-1231); the library uses its own
// implicit QL (sadmrg::tridiag_eig, symmetry-adapted-dmrg-library_b200/csrc/dmrg.cpp),
// exported by libsadmrg_b200.so.  This program draws seeded tridiagonals of the
// kinds a Lanczos run produces and some harder ones -- random alpha / positive
// beta, Wilkinson W+ (close eigenvalue pairs), a coupling exactly zero (split
// matrix), scaled by 1e-150 and 1e+150 -- and compares:
//   eigenvalues (ascending) with dstev's, to 1e-13 n |T|;
//   the residual |T z - l z| and the orthogonality of the library's vectors;
//   the ground-state vector (the one the Lanczos uses) with dstev's up to sign,
//   where the gap to the next eigenvalue exceeds 1e-6 |T|.
//
// usage: tridiag_check <cases> <seed>
// prints: cases, largest eigenvalue error, residual, orthogonality and ground
// vector errors (all relative to |T|), mismatches; exits 1 on any mismatch.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

namespace sadmrg {
void tridiag_eig(int n, std::vector<double>& d, std::vector<double> e, std::vector<double>& z);
}
extern "C" void dstev_(const char* jobz, const int* n, double* d, double* e, double* z, const int* ldz, double* work,
                       int* info);

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: tridiag_check <cases> <seed>\n");
    return 2;
  }
  const int cases = std::atoi(argv[1]);
  std::mt19937_64 rng((unsigned long long)std::atoll(argv[2]));
  std::normal_distribution<double> nd(0.0, 1.0);
  double ev_err = 0.0, res_err = 0.0, orth_err = 0.0, gs_err = 0.0;
  long bad = 0, gs_checked = 0;
  for (int c = 0; c < cases; ++c) {
    const int kind = c % 4;
    const int n = 1 + (int)(rng() % 100);
    std::vector<double> d(n), e(n > 1 ? n - 1 : 0);
    if (kind == 1) {   // Wilkinson W+: d_i = |i - m|, e = 1
      for (int i = 0; i < n; ++i) d[i] = std::fabs(i - (n - 1) / 2.0);
      for (auto& x : e) x = 1.0;
    } else {
      for (auto& x : d) x = nd(rng);
      for (auto& x : e) x = std::fabs(nd(rng)) + 1e-3;
      if (kind == 2 && n > 2) e[rng() % (n - 1)] = 0.0;   // split matrix
    }
    const double scale = (c % 7 == 5) ? 1e-150 : (c % 7 == 6) ? 1e150 : 1.0;
    double tn = 0.0;
    for (int i = 0; i < n; ++i) {
      d[i] *= scale;
      tn = std::max(tn, std::fabs(d[i]));
    }
    for (auto& x : e) {
      x *= scale;
      tn = std::max(tn, std::fabs(x));
    }
    if (tn == 0.0) tn = 1.0;

    // the library
    std::vector<double> dl = d, z;
    sadmrg::tridiag_eig(n, dl, e, z);
    // LAPACK, as the reference calls it
    std::vector<double> dr = d, er = e, zr((size_t)n * n), work(std::max(1, 2 * n - 2));
    er.resize(std::max(1, n), 0.0);
    int info = 0;
    const char jobz = 'V';
    dstev_(&jobz, &n, dr.data(), er.data(), zr.data(), &n, work.data(), &info);
    if (info != 0) { ++bad; continue; }

    bool ok = true;
    for (int i = 0; i < n; ++i) {
      const double err = std::fabs(dl[i] - dr[i]) / tn;
      ev_err = std::max(ev_err, err);
      if (err > 1e-13 * n) ok = false;
      if (i && dl[i] < dl[i - 1]) ok = false;
    }
    for (int k = 0; k < n; ++k) {
      const double* v = &z[(size_t)k * n];
      double r = 0.0;
      for (int i = 0; i < n; ++i) {
        double t = d[i] * v[i] - dl[k] * v[i];
        if (i > 0) t += e[i - 1] * v[i - 1];
        if (i < n - 1) t += e[i] * v[i + 1];
        r = std::max(r, std::fabs(t));
      }
      res_err = std::max(res_err, r / tn);
      if (r / tn > 1e-13 * n) ok = false;
      for (int l = k; l < n; ++l) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += v[i] * z[(size_t)l * n + i];
        const double o = std::fabs(s - (l == k ? 1.0 : 0.0));
        orth_err = std::max(orth_err, o);
        if (o > 1e-13 * n) ok = false;
      }
    }
    if (n == 1 || (dr[1] - dr[0]) > 1e-6 * tn) {
      ++gs_checked;
      double s = 0.0;
      for (int i = 0; i < n; ++i) s += z[i] * zr[i];
      const double sg = s >= 0.0 ? 1.0 : -1.0;
      double g = 0.0;
      for (int i = 0; i < n; ++i) g = std::max(g, std::fabs(z[i] - sg * zr[i]));
      gs_err = std::max(gs_err, g);
      if (g > 1e-9) ok = false;
    }
    if (!ok) ++bad;
  }
  std::printf("cases %d ev_err %.3e residual %.3e orth %.3e ground_vec %.3e ground_checked %ld mismatches %ld\n",
              cases, ev_err, res_err, orth_err, gs_err, gs_checked, bad);
  return bad ? 1 : 0;
}
