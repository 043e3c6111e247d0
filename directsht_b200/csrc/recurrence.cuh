// The FP64 Ylm / dYlm recurrences of one column m at one node x, step by step in l.
//
// Shared by the table build (tables.cu) and by the kernels that regenerate table values on
// the fly (heavy.cu), so both produce bitwise the same numbers.  Every product and sum is a
// separately rounded __dmul_rn / __dadd_rn / __ddiv_rn in the order of the reference's
// numpy/numba path:
//   Y_mm        = prod_{k=1..m} (-sqrt(1 - 1/2k) sx)              sht/legendre_py.py:28-30
//   Y_{m+1,m}   = sqrt(2m+1) x Y_mm   (m = 0: x)                  sht/legendre_py.py:32-34
//   Y_lm        = ((2l-1) x Y_{l-1} - (l+m-1) Y_{l-2} f2) q        sht/legendre_py.py:98-100
//   dY_l0       = l/(1-x^2) (Y_{l-1} - x Y_l)                     sht/legendre_py.py:56
//   dY_lm       = ((l+m) f1 Y_{l-1} - l x Y_l) / (1-x^2)          sht/legendre_py.py:115-116
// with f2 = sqrt((l-m-1)/(l+m-1)), f1 = sqrt((l-m)/(l+m)), q = f1/(l-m); both values are then
// scaled by nrm = sqrt((2l+1)/4pi) (sht/legendre_py.py:67-82).
#pragma once

#include "dsht_internal.cuh"

namespace dsht {

// Per-l coefficients of the column m:
//   a = 2l-1, b = l+m-1, f2, q, dc = (l+m) f1, nrm.
struct Coef {
  double a, b, f2, q, dc, nrm;
};

__device__ __forceinline__ Coef make_coef(int l, int m) {
  Coef c;
  c.a = (double)(2 * l - 1);
  c.b = (double)(l + m - 1);
  c.f2 = (l >= m + 2) ? sqrt((double)(l - m - 1) / (double)(l + m - 1)) : 0.0;
  const double f1 = (l > m) ? sqrt((double)(l - m) / (double)(l + m)) : 0.0;
  c.q = (l > m) ? f1 / (double)(l - m) : 0.0;
  c.dc = (double)(l + m) * f1;
  c.nrm = sqrt((double)(2 * l + 1) / 4.0 / M_PI);
  return c;
}

// sqrt(1 - 1/2k), the diagonal factor of Y_kk / Y_{k-1,k-1} (k >= 1).
__device__ __forceinline__ double diag_factor(int k) { return sqrt(1.0 - 1.0 / (double)(2 * k)); }

// State of one (m, x) walk: the node's x, 1 - x^2, and the two previous rows.
struct ColumnState {
  double x, omx2;
  double y1, y2;  // Y_{l-1}, Y_{l-2} (unnormalised)
};

// x = j * step as numpy builds the grid; returns 1 - x^2 and sqrt(1 - x^2) = sx.
__device__ __forceinline__ void node_x(int j, double step, double* x, double* omx2, double* sx) {
  *x = (double)j * step;
  const double x2 = __dmul_rn(*x, *x);
  *omx2 = __dadd_rn(1.0, -x2);
  *sx = sqrt(*omx2);
}

// Y_mm from the diagonal factors smm[1..m].
__device__ __forceinline__ double diag_value(int m, double sx, const double* smm) {
  double ymm = 1.0;
  for (int k = 1; k <= m; ++k) ymm = __dmul_rn(__dmul_rn(-smm[k], sx), ymm);
  return ymm;
}

// Row l = m: (Y, dY) unnormalised; sets up the state.
__device__ __forceinline__ void column_first(int m, double x, double omx2, double ymm, ColumnState* st, double* y,
                                             double* d) {
  st->x = x;
  st->omx2 = omx2;
  *y = ymm;
  if (m == 0) {
    *d = 0.0;
  } else {  // ((l+m) f1) Y_{l-1} with f1 = 0, minus (l x) Y_l, over 1-x^2
    *d = __ddiv_rn(__dadd_rn(0.0, -__dmul_rn(__dmul_rn((double)m, x), ymm)), omx2);
  }
  st->y2 = 0.0;
  st->y1 = ymm;
}

// Row l = m + 1 (c = coefficients of l); advances the state.
__device__ __forceinline__ void column_second(int m, const Coef& c, ColumnState* st, double* y, double* d) {
  const int l = m + 1;
  const double x = st->x;
  if (m == 0) {
    *y = x;
    *d = 1.0;
  } else {
    *y = __dmul_rn(__dmul_rn(sqrt(2.0 * m + 1.0), x), st->y1);
    *d = __ddiv_rn(__dadd_rn(__dmul_rn(c.dc, st->y1), -__dmul_rn(__dmul_rn((double)l, x), *y)), st->omx2);
  }
  st->y2 = st->y1;
  st->y1 = *y;
}

// Row l >= m + 2 (c = coefficients of l); advances the state.
__device__ __forceinline__ void column_step(int m, int l, const Coef& c, ColumnState* st, double* y, double* d) {
  const double x = st->x;
  const double t = __dadd_rn(__dmul_rn(__dmul_rn(c.a, x), st->y1), -__dmul_rn(__dmul_rn(c.b, st->y2), c.f2));
  *y = __dmul_rn(t, c.q);
  if (m == 0) {
    *d = __dmul_rn(__ddiv_rn((double)l, st->omx2), __dadd_rn(st->y1, -__dmul_rn(x, *y)));
  } else {
    *d = __ddiv_rn(__dadd_rn(__dmul_rn(c.dc, st->y1), -__dmul_rn(__dmul_rn((double)l, x), *y)), st->omx2);
  }
  st->y2 = st->y1;
  st->y1 = *y;
}

}  // namespace dsht
