// Host build of the pencil algebra of step 3 (the same source the kernels
// run), exported for the CPU unit tests that compare it with the
// reference's setmacrhs/trid/dcheb.  Not part of the device library.
#include "fft.cuh"
#include "step3.cuh"

using namespace sb;

extern "C" void sbh_tau_solve(double lam, int n, int m, const double* f, double* x, const double* bc1,
                              const double* bc2, double* cp, double* wt) {
  // columns are contiguous vectors of n doubles; m <= 5
  Col F[5], X[5];
  for (int q = 0; q < m; ++q) {
    F[q] = Col{const_cast<double*>(f) + (size_t)q * n, 1};
    X[q] = Col{x + (size_t)q * n, 1};
  }
  Col C{cp, 1}, W{wt, 1};
  switch (m) {
    case 1: tau_solve<1>(lam, n, F, X, bc1, bc2, C, W); break;
    case 2: tau_solve<2>(lam, n, F, X, bc1, bc2, C, W); break;
    case 3: tau_solve<3>(lam, n, F, X, bc1, bc2, C, W); break;
    case 4: tau_solve<4>(lam, n, F, X, bc1, bc2, C, W); break;
    default: tau_solve<5>(lam, n, F, X, bc1, bc2, C, W); break;
  }
}

extern "C" void sbh_cheb_deriv(const double* a, double* b, int n) {
  cheb_deriv(Col{b, 1}, Col{const_cast<double*>(a), 1}, n);
}

// Host run of the shared-memory FFT passes on B interleaved columns
// (element i of column b at [i*B + b]); in/out complex interleaved.
extern "C" int sbh_fft(int n, const double* in, double* out, int sign) {
  const FFTPlan plan = fft_make_plan(n);
  if (plan.npass < 0) return -1;
  double2* tw = new double2[n];
  for (int m = 0; m < n; ++m) {
    long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
    tw[m] = double2{(double)cosl(ang), (double)sinl(ang)};
  }
  double2* a = new double2[n];
  double2* b = new double2[n];
  for (int i = 0; i < n; ++i) a[i] = double2{in[2 * i], in[2 * i + 1]};
  double2* src = a;
  double2* dst = b;
  for (int p = 0; p < plan.npass; ++p) {
    fft_pass<double, 1>(src, dst, plan, p, tw, sign, 0, 1);
    double2* t = src;
    src = dst;
    dst = t;
  }
  for (int i = 0; i < n; ++i) {
    out[2 * i] = src[i].x;
    out[2 * i + 1] = src[i].y;
  }
  delete[] a;
  delete[] b;
  delete[] tw;
  return plan.npass;
}
