// Host build of the pencil algebra of step 3 (the same source the kernels
// run), exported for the CPU unit tests that compare it with the
// reference's setmacrhs/trid/dcheb.  Not part of the device library.
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
