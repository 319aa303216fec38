/*
 * zdot_shim.c -- link-time shim for the reference CPU build (test infrastructure).
 *
 * The reference declares the complex BLAS dots with a result-pointer first
 * argument (scalar.hpp:44-45, called at scalar.hpp:161,169).  The OpenBLAS that
 * ships in this image is built with gfortran, which returns complex(8) by value,
 * so the reference's complex targets read garbage (E = 0 / NaN).  Defining the
 * two symbols here, with the signature the reference expects, makes the
 * executable's own definitions win over the shared library's.
 *
 * Semantics are the BLAS ones: zdotc = sum conj(x_i) * y_i, zdotu = sum x_i*y_i.
 */
#include <complex.h>

void zdotc_(double _Complex *res, const int *n, const double _Complex *x,
            const int *incx, const double _Complex *y, const int *incy) {
  double _Complex s = 0;
  for (int i = 0; i < *n; ++i) s += conj(x[i * (*incx)]) * y[i * (*incy)];
  *res = s;
}

void zdotu_(double _Complex *res, const int *n, const double _Complex *x,
            const int *incx, const double _Complex *y, const int *incy) {
  double _Complex s = 0;
  for (int i = 0; i < *n; ++i) s += x[i * (*incx)] * y[i * (*incy)];
  *res = s;
}
