// Filters of the ADM-RT large-eddy model (relaxation term, iles = 1): host
// set-up of the tables that the device kernels of les.cuh use.
//
// The model (bla/bla.f:1489-1518, bla/init_filter.f, bla/linearbl.f:1871-
// 1960, bla/nonlinbl.f:920-965) needs the high-pass filtered velocity
//   ihighorder = 2 (reference default):  gu = u - L_xz (I - H_y^(N+1)) u
//   ihighorder = 1:                      gu = (I - F_xz L_y)^(N+1) u
//   ihighorder = 0:                      gu = (1 - L_xz) u
// with, in the wall-normal direction, the implicit five-point filter
//   A f = B u   (low pass L_y = A^-1 B,  high pass H_y = I - L_y)
// on the Gauss-Lobatto points, and in x/z the same filter's transfer function
// on a uniform grid, F_xz(kx,kz) = G(kx) G(kz) and L_xz = 1 - (1 - F_xz)^(N+1).
//
// Each five-point explicit stencil b (offsets x_j from the centre point,
// index offsets s_j) satisfies
//   sum b_j = 1,  sum b_j x_j = 0,  sum b_j x_j^2 = 0   (second-order moments)
//   sum b_j (-1)^s_j = 0                                (zero response at the
//                                                        grid Nyquist number)
// and, for the one remaining degree of freedom,
//   interior (centred) rows: minimum dispersion, i.e. the smallest
//     (b_2 - b_-2)^2 + (b_1 - b_-1)^2 (the integral over [0, pi] of the
//     squared imaginary part of the index-space transfer function);
//   rows 2 and ny-1 (one point on one side, three on the other):
//     sum b_j x_j^3 = 0.
// The implicit stencil a is a_j = r b_j off the centre, a_0 = 1 - sum a_j,
// with r the root -(beta + sqrt(beta^2 - 4 alpha gamma)) / (2 alpha) of the
// condition |E / I| = 1/2 at the cut-off k = pi * cutoff, E and I the
// index-space transfer functions of b and a (I = 1 - r + r E).  Rows 1 and ny
// are not filtered.  Rows 2 and ny-1 reach five points on one side; one step
// of elimination with rows 3 and ny-2 makes A pentadiagonal, and the same
// combination is applied to the right-hand side.
//
// The moment conditions are solved here as small linear systems in long
// double; the coefficients agree with the reference's closed forms to
// rounding.
#pragma once

#include <cmath>
#include <vector>

namespace sb {

struct LesFilter {
  int nyp = 0, nx2 = 0, nz = 0, iord = 0;
  std::vector<double> g1, g2;   // [nyp][5] explicit and implicit stencils (reference gewy1, gewy2)
  std::vector<double> specx;    // [nx/2 + 1] G at kx = 0..nx/2 (gewspecx)
  std::vector<double> specz;    // [nz/2 + 1] G at kz = 0..nz/2 (gewspecz)
  std::vector<double> filtxz;   // [nz][nx/2] F_xz
  std::vector<double> lpfxz;    // [nz][nx/2] L_xz
  double fact2 = 0, factm2 = 0; // row-2 / row-(ny-1) elimination factors
  // LU factors of A (no pivoting): row j of A = (e, f, g, h, k) at columns
  // j-2..j+2; L has e, l1 and the pivots d; U is unit upper with u1, u2.
  std::vector<double> e, l1, dinv, u1, u2;
};

namespace les_detail {

// Gaussian elimination with partial pivoting, n <= 6, in long double.
inline bool solve_small(int n, long double* a /* n x n row-major */, long double* b) {
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (fabsl(a[r * n + c]) > fabsl(a[p * n + c])) p = r;
    if (a[p * n + c] == 0.0L) return false;
    if (p != c) {
      for (int k = 0; k < n; ++k) {
        long double t = a[c * n + k];
        a[c * n + k] = a[p * n + k];
        a[p * n + k] = t;
      }
      long double t = b[c];
      b[c] = b[p];
      b[p] = t;
    }
    for (int r = c + 1; r < n; ++r) {
      const long double m = a[r * n + c] / a[c * n + c];
      if (m == 0.0L) continue;
      for (int k = c; k < n; ++k) a[r * n + k] -= m * a[c * n + k];
      b[r] -= m * b[c];
    }
  }
  for (int r = n - 1; r >= 0; --r) {
    long double s = b[r];
    for (int k = r + 1; k < n; ++k) s -= a[r * n + k] * b[k];
    b[r] = s / a[r * n + r];
  }
  return true;
}

// Rows of the four common conditions for offsets x[5], index offsets s[5].
inline void common_rows(const long double* x, const int* s, long double* a, long double* b) {
  for (int j = 0; j < 5; ++j) {
    a[0 * 5 + j] = 1.0L;
    a[1 * 5 + j] = x[j];
    a[2 * 5 + j] = x[j] * x[j];
    a[3 * 5 + j] = (s[j] & 1) ? -1.0L : 1.0L;
  }
  b[0] = 1.0L;
  b[1] = b[2] = b[3] = 0.0L;
}

// Explicit stencil with the third moment zero (rows 2 and ny-1).
inline bool explicit_m3(const long double* x, const int* s, long double* out) {
  long double a[25], b[5];
  common_rows(x, s, a, b);
  for (int j = 0; j < 5; ++j) a[4 * 5 + j] = x[j] * x[j] * x[j];
  b[4] = 0.0L;
  if (!solve_small(5, a, b)) return false;
  for (int j = 0; j < 5; ++j) out[j] = b[j];
  return true;
}

// Centred explicit stencil of minimum index-space dispersion: the family
// c(t) = c0 + t n of the four conditions, parametrised by its last weight,
// and the t minimising (c4 - c0)^2 + (c3 - c1)^2.
inline bool explicit_mindisp(const long double* x, const int* s, long double* out) {
  long double c[2][5];
  for (int t = 0; t < 2; ++t) {
    long double a[25], b[5];
    common_rows(x, s, a, b);
    for (int j = 0; j < 5; ++j) a[4 * 5 + j] = (j == 4) ? 1.0L : 0.0L;
    b[4] = (long double)t;
    if (!solve_small(5, a, b)) return false;
    for (int j = 0; j < 5; ++j) c[t][j] = b[j];
  }
  long double n[5];
  for (int j = 0; j < 5; ++j) n[j] = c[1][j] - c[0][j];
  const long double w0 = c[0][4] - c[0][0], w1 = c[0][3] - c[0][1];
  const long double v0 = n[4] - n[0], v1 = n[3] - n[1];
  const long double den = v0 * v0 + v1 * v1;
  const long double t = den > 0.0L ? -(w0 * v0 + w1 * v1) / den : 0.0L;
  for (int j = 0; j < 5; ++j) out[j] = c[0][j] + t * n[j];
  return true;
}

// Implicit stencil from the explicit one (index offsets s, centre index ic).
inline void implicit_from(const long double* bx, const int* s, int ic, double cutoff, long double* out) {
  const long double pi = 4.0L * atanl(1.0L);
  const long double rk = pi * (long double)cutoff;
  long double gre = 0.0L, gim = 0.0L;
  for (int j = 0; j < 5; ++j) {
    gre += bx[j] * cosl((long double)s[j] * rk);
    gim += bx[j] * sinl((long double)s[j] * rk);
  }
  const long double al = (gre - 1.0L) * (gre - 1.0L) + gim * gim;
  const long double be = 2.0L * (gre - 1.0L);
  const long double ga = 1.0L - 4.0L * gre * gre - 4.0L * gim * gim;
  const long double r = (-be - sqrtl(be * be - 4.0L * al * ga)) / (2.0L * al);
  long double sum = 0.0L;
  for (int j = 0; j < 5; ++j)
    if (j != ic) {
      out[j] = r * bx[j];
      sum += out[j];
    }
  out[ic] = 1.0L - sum;
}

// Real part of E/I on a uniform grid at index wavenumber k (centred stencils).
inline double transfer(const long double* bx, const long double* ax, long double k) {
  long double ra = 0, rb = 0, rc = 0, rd = 0;
  for (int j = 0; j < 5; ++j) {
    const long double sj = (long double)(j - 2);
    ra += bx[j] * cosl(sj * k);
    rb += bx[j] * sinl(sj * k);
    rc += ax[j] * cosl(sj * k);
    rd += ax[j] * sinl(sj * k);
  }
  return (double)((ra * rc + rb * rd) / (rc * rc + rd * rd));
}

}  // namespace les_detail

// Pentadiagonal A from the implicit stencils (rows 2 and ny-1 combined with
// rows 3 and ny-2) and its LU factors.
inline bool les_filter_factor(LesFilter& F) {
  const int n = F.nyp;
  auto G = [&](int row, int l) -> long double { return (long double)F.g2[(size_t)row * 5 + l]; };
  std::vector<long double> e(n, 0), f(n, 0), g(n, 0), h(n, 0), k(n, 0);
  g[0] = 1;
  g[n - 1] = 1;
  const long double fa = -G(1, 4) / G(2, 4);
  const long double fb = -G(n - 2, 0) / G(n - 3, 0);
  F.fact2 = (double)fa;
  F.factm2 = (double)fb;
  f[1] = G(1, 0) + G(2, 0) * fa;
  g[1] = G(1, 1) + G(2, 1) * fa;
  h[1] = G(1, 2) + G(2, 2) * fa;
  k[1] = G(1, 3) + G(2, 3) * fa;
  for (int j = 2; j <= n - 3; ++j) {
    e[j] = G(j, 0);
    f[j] = G(j, 1);
    g[j] = G(j, 2);
    h[j] = G(j, 3);
    k[j] = G(j, 4);
  }
  e[n - 2] = G(n - 2, 1) + G(n - 3, 1) * fb;
  f[n - 2] = G(n - 2, 2) + G(n - 3, 2) * fb;
  g[n - 2] = G(n - 2, 3) + G(n - 3, 3) * fb;
  h[n - 2] = G(n - 2, 4) + G(n - 3, 4) * fb;
  std::vector<long double> l1(n, 0), d(n, 0), u1(n, 0), u2(n, 0);
  for (int j = 0; j < n; ++j) {
    l1[j] = f[j] - (j >= 2 ? e[j] * u1[j - 2] : 0.0L);
    d[j] = g[j] - (j >= 2 ? e[j] * u2[j - 2] : 0.0L) - (j >= 1 ? l1[j] * u1[j - 1] : 0.0L);
    if (d[j] == 0.0L) return false;
    u1[j] = (h[j] - (j >= 1 ? l1[j] * u2[j - 1] : 0.0L)) / d[j];
    u2[j] = k[j] / d[j];
  }
  F.e.resize(n);
  F.l1.resize(n);
  F.dinv.resize(n);
  F.u1.resize(n);
  F.u2.resize(n);
  for (int j = 0; j < n; ++j) {
    F.e[j] = (double)e[j];
    F.l1[j] = (double)l1[j];
    F.dinv[j] = (double)(1.0L / d[j]);
    F.u1[j] = (double)u1[j];
    F.u2[j] = (double)u2[j];
  }
  return true;
}

// Builds the tables for nyp Gauss-Lobatto points y_j = 1 + cos(pi j/(nyp-1))
// (the reference's gridy with dstar = 1), nx/2 x nz stored modes, cut-off
// wavenumber fraction cutoff = 1/cutoff_inv and order N = iord.  Returns
// false on a singular condition system (not reached for nyp >= 7).
// secondary: the filter of the dynamic HPF model (bla/bla.f:1520-1545): the
// x and z transfer functions span kx = 0..nx/4 and kz = 0..nz/4 (the
// reference's init_filter called with nx/4+1, nz/4+1 points) and are zero
// above; the wall-normal stencils do not depend on it.
inline bool les_filter_build(int nyp, int nx, int nz, double cutoff, int iord, LesFilter& F,
                             bool secondary = false) {
  using namespace les_detail;
  if (nyp < 7 || (nyp % 2) == 0 || nx < 2 || nz < 2 || iord < 0) return false;
  F.nyp = nyp;
  F.nx2 = nx / 2;
  F.nz = nz;
  F.iord = iord;
  F.g1.assign((size_t)nyp * 5, 0.0);
  F.g2.assign((size_t)nyp * 5, 0.0);
  const long double pi = 4.0L * atanl(1.0L);
  std::vector<long double> y(nyp);
  for (int j = 0; j < nyp; ++j) y[j] = 1.0L + cosl(pi * (long double)j / (long double)(nyp - 1));
  // homogeneous (uniform grid) stencil for x and z
  {
    const long double x[5] = {-2, -1, 0, 1, 2};
    const int s[5] = {-2, -1, 0, 1, 2};
    long double bx[5], ax[5];
    if (!explicit_mindisp(x, s, bx)) return false;
    implicit_from(bx, s, 2, cutoff, ax);
    const int nxs = (secondary ? nx / 4 : nx / 2) + 1, nzs = (secondary ? nz / 4 : nz / 2) + 1;
    F.specx.assign(nx / 2 + 1, 0.0);
    F.specz.assign(nz / 2 + 1, 0.0);
    for (int i = 0; i < nxs; ++i) F.specx[i] = transfer(bx, ax, (long double)i * pi / (long double)(nxs - 1));
    for (int i = 0; i < nzs; ++i) F.specz[i] = transfer(bx, ax, (long double)i * pi / (long double)(nzs - 1));
  }
  // wall-normal stencils; the distances are measured as in the reference:
  // positive towards larger index, y decreasing with the index
  auto put = [&](int row, const long double* bx, const long double* ax) {
    for (int l = 0; l < 5; ++l) {
      F.g1[(size_t)row * 5 + l] = (double)bx[l];
      F.g2[(size_t)row * 5 + l] = (double)ax[l];
    }
  };
  {
    // row 1 (0-based 0) and row nyp: identity in slot 1 and slot 5
    F.g1[0] = F.g2[0] = 1.0;
    F.g1[(size_t)(nyp - 1) * 5 + 4] = F.g2[(size_t)(nyp - 1) * 5 + 4] = 1.0;
  }
  {
    // row 2: points 1..5, centre 2
    const int k = 1;
    long double x[5], bx[5], ax[5];
    const int s[5] = {-1, 0, 1, 2, 3};
    for (int l = 0; l < 5; ++l) x[l] = y[k] - y[l];
    if (!explicit_m3(x, s, bx)) return false;
    implicit_from(bx, s, 1, cutoff, ax);
    put(k, bx, ax);
  }
  for (int k = 2; k <= nyp - 3; ++k) {
    long double x[5], bx[5], ax[5];
    const int s[5] = {-2, -1, 0, 1, 2};
    for (int l = 0; l < 5; ++l) x[l] = y[k] - y[k - 2 + l];
    if (!explicit_mindisp(x, s, bx)) return false;
    implicit_from(bx, s, 2, cutoff, ax);
    put(k, bx, ax);
  }
  {
    // row nyp-1: points nyp-4..nyp, centre nyp-1
    const int k = nyp - 2;
    long double x[5], bx[5], ax[5];
    const int s[5] = {-3, -2, -1, 0, 1};
    for (int l = 0; l < 5; ++l) x[l] = y[k] - y[k - 3 + l];
    if (!explicit_m3(x, s, bx)) return false;
    implicit_from(bx, s, 3, cutoff, ax);
    put(k, bx, ax);
  }
  // x/z tables in the device order [kz][kx]
  F.filtxz.assign((size_t)nz * F.nx2, 0.0);
  F.lpfxz.assign((size_t)nz * F.nx2, 0.0);
  for (int iz = 0; iz < nz; ++iz) {
    const double gz = (iz <= nz / 2 - 1) ? F.specz[iz] : F.specz[nz - iz];
    for (int kx = 0; kx < F.nx2; ++kx) {
      const double f = F.specx[kx] * gz;
      double q = 1.0;
      for (int i = 0; i <= iord; ++i) q *= (1.0 - f);
      F.filtxz[(size_t)iz * F.nx2 + kx] = f;
      F.lpfxz[(size_t)iz * F.nx2 + kx] = 1.0 - q;
    }
  }
  return les_filter_factor(F);
}

// Per-row device table (les.cuh: LES_ROW doubles per row).
inline void les_filter_rows(const LesFilter& F, std::vector<double>& out) {
  const int n = F.nyp;
  out.assign((size_t)n * 15, 0.0);
  for (int j = 0; j < n; ++j) {
    double* r = &out[(size_t)j * 15];
    for (int l = 0; l < 5; ++l) {
      r[l] = F.g2[(size_t)j * 5 + l] - F.g1[(size_t)j * 5 + l];
      r[5 + l] = F.g1[(size_t)j * 5 + l];
    }
    r[10] = F.e[j];
    r[11] = F.l1[j];
    r[12] = F.dinv[j];
    r[13] = F.u1[j];
    r[14] = F.u2[j];
  }
}

}  // namespace sb
