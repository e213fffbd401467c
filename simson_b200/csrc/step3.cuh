// Step 3 of the RK substep: implicit Chebyshev-tau solves per (kx,kz) pencil
// (the work bla/linearbl.f does per xy-plane), plus the startup partial
// right-hand side (bla/prhs.f).
//
// Chebyshev transforms (k_cheb): physical <-> Chebyshev along y as a DCT-I of
// length N+1 (N = ny-1), computed as a complex FFT of the even extension of
// length 2N in shared memory over a tile of PB pencils.  Conventions are the
// reference's (bla/cvecfft_acc.f vchbf/vchbb with the normalisation of
// linearbl.f:262): a_k = 2/(N cbar_k) sum_j u_j cos(pi jk/N)/cbar_j,
// u_j = sum_k a_k cos(pi jk/N), cbar_0 = cbar_N = 2, else 1.
//
// Pencil algebra (k_pencil, one thread per complex pencil, columns strided by
// NP so a warp's accesses coalesce): the tau method of Canuto et al. for
// (D^2 - lambda) psi = f (bla/setmacrhs.f, bla/trid.f:120-200), the
// velocity-vorticity recovery and the next partial right-hand side, in the
// order linearbl.f:257-1860 uses for the channel (ibc = 0, tau).
#pragma once
#include <type_traits>

#include "fft.cuh"
#include "layout.cuh"

namespace sb {

#ifndef SB_HD
#define SB_HD __host__ __device__
#endif

template <class S>
struct ColT {
  S* a;
  size_t s;
  SB_HD __forceinline__ S& operator[](int j) const { return a[(size_t)j * s]; }
};
typedef ColT<double> Col;

// L2 prefetch of a row a few iterations ahead of a sweep: the sweeps are
// serial in y, so without it each row's loads wait a full DRAM latency.
// The prefetch holds no register; callers pass in-range addresses only, and
// addresses outside the global window (the mean-flow solve keeps its columns
// in shared memory) are skipped.
#ifndef SB_PF_ROWS
#define SB_PF_ROWS 3
#endif
SB_HD __forceinline__ void pf_l2(const void* ptr) {
#ifdef __CUDA_ARCH__
  if (__isGlobal(ptr)) asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(ptr)));
#else
  (void)ptr;
#endif
}

__device__ __forceinline__ Col col_re(double2* arr, int p, int NP) { return Col{reinterpret_cast<double*>(arr) + 2 * (size_t)p, 2 * (size_t)NP}; }
__device__ __forceinline__ Col col_im(double2* arr, int p, int NP) { return Col{reinterpret_cast<double*>(arr) + 2 * (size_t)p + 1, 2 * (size_t)NP}; }
__device__ __forceinline__ Col col_r(double* arr, int p, int NP) { return Col{arr + p, (size_t)NP}; }

// Chebyshev derivative: b = D a, by the backward recurrence
// b_j = b_{j+2} + 2(j+1) a_{j+1}, b_{n-1} = 0, b_0 halved (bla/dcheb.f).
SB_HD inline void cheb_deriv(Col b, Col a, int n) {
  // a and b never alias: loads may run ahead of the stores
  const double* __restrict__ ap = a.a;
  double* __restrict__ bp = b.a;
  const size_t sa = a.s, sb = b.s;
  double bp2 = 2.0 * (double)(n - 1) * ap[(size_t)(n - 1) * sa];  // b[n-2]
  double bp1 = 2.0 * (double)(n - 2) * ap[(size_t)(n - 2) * sa];  // b[n-3]
  bp[(size_t)(n - 2) * sb] = bp2;
  bp[(size_t)(n - 3) * sb] = bp1;
#pragma unroll 8
  for (int j = n - 4; j >= 0; --j) {
    if (j + 1 - SB_PF_ROWS >= 0) pf_l2(ap + (size_t)(j + 1 - SB_PF_ROWS) * sa);
    const double v = bp2 + 2.0 * (double)(j + 1) * ap[(size_t)(j + 1) * sa];
    bp2 = bp1;
    bp1 = v;
    bp[(size_t)j * sb] = (j == 0) ? 0.5 * v : v;
  }
  bp[(size_t)(n - 1) * sb] = 0.0;
}

// The lam-independent factors of the tau rows (bla/setmacrhs.f) and of the
// tau right-hand side, per 1-based row index i, as FP64 tables: IEEE
// division is correctly rounded, so an entry equals the quotient computed in
// place and the solves keep their arithmetic bit for bit, without the FP64
// divisions in their serial sweeps.  Rows from TAU_TAB_N on are computed.
constexpr int TAU_TAB_N = 640;
// The FP32 instance (the mixed path's omega_y / phi solve) takes its own
// table of the same quotients evaluated in FP32.
template <class S>
struct TauTab {
  S c[TAU_TAB_N];   // -0.25 (i = 1), -0.25 / (i (i + 1))
  S d[TAU_TAB_N];   // 0.5 / (i (i + 2))
  S e[TAU_TAB_N];   // -0.25 / ((i + 1)(i + 2))
  S ra[TAU_TAB_N];  // 0.25 / ((i - 2)(i - 1)), i >= 4 (0 below)
  S rb[TAU_TAB_N];  // -0.5 / ((i - 2) i), i >= 3
  S rc[TAU_TAB_N];  // 0.25 / ((i - 1) i), i >= 2
};
template <class S>
constexpr TauTab<S> tau_tab_make() {
  TauTab<S> t{};
  for (int i = 1; i < TAU_TAB_N; ++i) {
    const S di = (S)i;
    t.c[i] = (i == 1) ? (S)-0.25 : (S)-0.25 / (di * (di + (S)1.0));
    t.d[i] = (S)0.5 / (di * (di + (S)2.0));
    t.e[i] = (S)-0.25 / ((di + (S)1.0) * (di + (S)2.0));
    t.ra[i] = (i >= 4) ? (S)0.25 / ((di - (S)2.0) * (di - (S)1.0)) : (S)0.0;
    t.rb[i] = (i >= 3) ? (S)-0.5 / ((di - (S)2.0) * di) : (S)0.0;
    t.rc[i] = (i >= 2) ? (S)0.25 / ((di - (S)1.0) * di) : (S)0.0;
  }
  return t;
}
inline constexpr TauTab<double> kTauHost = tau_tab_make<double>();
inline constexpr TauTab<float> kTauHostF = tau_tab_make<float>();
#ifdef __CUDACC__
// read with one row index per warp at a time (the thread-per-pencil sweeps):
// constant-cache broadcasts
__constant__ const TauTab<double> kTauConst = tau_tab_make<double>();
__constant__ const TauTab<float> kTauConstF = tau_tab_make<float>();
// the same in global memory, for reads whose row index differs across a
// warp (the warp-per-pencil kernels: the constant cache would serialise them)
__device__ const TauTab<double> kTauGlobal = tau_tab_make<double>();
#endif
#ifdef __CUDA_ARCH__
#define SB_TAUTAB kTauConst
#define SB_TAUTAB_F kTauConstF
#else
#define SB_TAUTAB kTauHost
#define SB_TAUTAB_F kTauHostF
#endif
// the table of the solve's scalar type
template <class S>
SB_HD __forceinline__ const TauTab<S>& tau_tab();
template <>
SB_HD __forceinline__ const TauTab<double>& tau_tab<double>() { return SB_TAUTAB; }
template <>
SB_HD __forceinline__ const TauTab<float>& tau_tab<float>() { return SB_TAUTAB_F; }

// Tau-method coefficients of (D^2 - lam) for the quasi-tridiagonal rows
// (1-based row index i as in bla/setmacrhs.f).
template <class S>
SB_HD __forceinline__ S tau_c(int i, S lam) {
  if (i < TAU_TAB_N) return tau_tab<S>().c[i] * lam;
  return (i == 1) ? (S)-0.25 * lam : ((S)-0.25 / ((S)i * ((S)i + (S)1.0))) * lam;
}
template <class S>
SB_HD __forceinline__ S tau_d(int i, S lam) {
  if (i < TAU_TAB_N) return (S)1.0 + tau_tab<S>().d[i] * lam;
  return (S)1.0 + ((S)0.5 / ((S)i * ((S)i + (S)2.0))) * lam;
}
template <class S>
SB_HD __forceinline__ S tau_e(int i, S lam) {
  if (i < TAU_TAB_N) return tau_tab<S>().e[i] * lam;
  return ((S)-0.25 / (((S)i + (S)1.0) * ((S)i + (S)2.0))) * lam;
}

// Tau right-hand side of row i (3 <= i <= n, 1-based) from f: the
// Chebyshev-coefficient form of u'' = f + lam u, truncated at n modes.
SB_HD __forceinline__ double tau_rhs(const Col& f, int i, int n) {
  if (f.a == nullptr) return 0.0;
  auto F = [&](int k) { return f[k - 1]; };
  const double di = (double)i;
  if (i == 3) return 0.25 * F(1) + F(5) / 24.0 - F(3) / 6.0;
  double r = (0.25 / ((di - 2.0) * (di - 1.0))) * F(i - 2);
  if (i <= n - 2) r += (-0.5 / ((di - 2.0) * di)) * F(i);
  if (i <= n - 4) r += (0.25 / ((di - 1.0) * di)) * F(i + 2);
  return r;
}

// Solve (D^2 - lam) x_q = f_q, q < M, by the Chebyshev tau method with the
// boundary rows  sum_{k even} x_k = bc1[q],  sum_{k odd} x_k = bc2[q]
// (i.e. x(+1) = bc1+bc2, x(-1) = bc1-bc2).  The elimination is the one of
// bla/trid.f:120-200 -- upper off-diagonal from the top, the two full rows
// through the weights W, then the lower off-diagonal -- with the same rounding
// of every operation, reorganised into three sweeps whose recurrences run in
// registers:
//   1. backward (rows n..3): factor 1/d', c' = c/d'; eliminated right-hand side
//      x(i) = (rhs(i) - x(i+2) e(i-2)) / d'(i-2); weights W(i) = 1 - c'(i) W(i+2);
//   2. ascending boundary sums (same summation order as the reference);
//   3. forward (rows 3..n): x(i) -= c'(i-2) x(i-2).
// cp, wt: per-pencil scratch columns (n entries each).  f[q].a == nullptr
// means a zero right-hand side.
//
// FAST (the mixed-precision path): the boundary sums are accumulated during
// the backward sweep (descending order, W kept in registers, wt unused) and,
// if dsum != nullptr, the forward sweep also returns the parity sums of the
// derivative coefficients, dsum[q][0] = sum_{j even} (D x)_j =
// sum_{k odd} k^2 x_k and dsum[q][1] = sum_{j odd} (D x)_j = sum_{k even}
// k^2 x_k (D x at y = +-1), so no column of D x is formed.  Two column passes
// fewer per solution; the same arithmetic in a different summation order.
//
// pre (optional): called at the top of backward row i as pre(i, fnew) and
// returns in fnew[q] (type FS, the forcing's storage type) the right-hand
// side f(i-3) of every column (0-based rows; the caller has produced rows n-1
// and n-2 itself), so a right-hand side assembled row by row never goes
// through memory; f[] is then unused.
struct NoPre {};

//
// CPC: cp (and, for the reference order, wt) already hold this lam's
// coefficients, written by an earlier solve with the same lam and n: the
// backward sweep computes them in registers as always but does not store them.
template <int M, class S = double, class FS = S, bool FAST = false, bool CPC = false, class Pre = NoPre>
SB_HD void tau_solve(S lam, int n, const ColT<FS>* f, const ColT<S>* x, const S* bc1, const S* bc2, ColT<S> cp,
                     ColT<S> wt, S (*dsum)[2] = nullptr, Pre pre = Pre()) {
  constexpr bool HOOK = !std::is_same<Pre, NoPre>::value;
  // every column is a distinct array: restrict-qualified raw pointers let the
  // loads of a sweep run ahead of its stores
  const FS* __restrict__ fp[M];
  S* __restrict__ xp[M];
  size_t fs[M], xs[M];
#pragma unroll
  for (int q = 0; q < M; ++q) {
    fp[q] = HOOK ? nullptr : f[q].a;
    fs[q] = HOOK ? 0 : f[q].s;
    xp[q] = x[q].a;
    xs[q] = x[q].s;
  }
  S* __restrict__ cpp = cp.a;
  S* __restrict__ wtp = wt.a;
  const size_t cs = cp.s, ws = wt.s;
  S xa[M], xb[M];  // x computed 1 and 2 rows ago (x(i+1), x(i+2))
  S q1 = (S)0.0, q2 = (S)0.0;  // c' computed 1 and 2 rows ago: q2 = c'(i) at row i
  S w1 = (S)0.0, w2 = (S)0.0;  // W computed 1 and 2 rows ago: w2 = W(i+2) at row i
  S bs_odd[M], bs_even[M];  // FAST: boundary sums
#pragma unroll
  for (int q = 0; q < M; ++q) xa[q] = xb[q] = bs_odd[q] = bs_even[q] = (S)0.0;
  // right-hand-side window: row i reads f(i-3), f(i-1), f(i+1) (0-based);
  // per row parity the last two stay in registers, so each row loads one
  // value per column (row i-2 reuses f(i-1) and f(i-3)). Used by the FP64
  // path, with pre and (SB_TAU_WIN_ALL) in the reordered (FAST) variant: one
  // load per row instead of three (mixed pencil kernel 1.02 -> 1.005 ms, no
  // spill at its 128-register cap).  The window holds
  // the values in the forcing's storage type FS: they come from FS columns or
  // from pre, which rounds them to FS, so this is exact (and halves the
  // window's registers when FS is float).
#ifndef SB_TAU_WIN_ALL
#define SB_TAU_WIN_ALL 1
#endif
  constexpr bool WIN = !FAST || HOOK || SB_TAU_WIN_ALL;
  FS wlo0[M], whi0[M], wlo1[M], whi1[M];  // even / odd rows (selects keep them in registers)
#pragma unroll
  for (int q = 0; q < M; ++q) wlo0[q] = wlo1[q] = whi0[q] = whi1[q] = (FS)0.0;
  // FAST: f(i-3) of the window read one row early, before the row's stores
  // (the FP64 order keeps the plain load: one more live value spills there)
  constexpr bool EARLY = FAST && !HOOK;
  FS fpre[M];
#pragma unroll
  for (int q = 0; q < M; ++q) fpre[q] = (EARLY && fp[q] != nullptr) ? fp[q][(size_t)(n - 3) * fs[q]] : (FS)0.0;
  for (int i = n; i >= 3; --i) {
    const int pr = i & 1;
    FS fh[M];
    if constexpr (HOOK) pre(i, fh);
    S dinv = (S)1.0, cnew = (S)0.0, wnew = (S)0.0;
    if (i <= n - 2) {
      const int m = i - 2;  // factor row m (trid.f: d(m) = 1/(d(m) - c(m+2) e(m)))
      dinv = (i >= n - 3) ? (S)1.0 / tau_d(m, lam) : (S)1.0 / (tau_d(m, lam) - q2 * tau_e(m, lam));
      cnew = tau_c(m, lam) * dinv;
      if (!CPC) cpp[(size_t)(m - 1) * cs] = cnew;
      wnew = (i >= n - 3) ? (S)1.0 - tau_c(i, lam) : (S)1.0 - q2 * w2;
      if (!FAST && !CPC) wtp[(size_t)(i - 1) * ws] = wnew;
    }
    const S di = (S)i;
    S ca, cb, cc;
    if (i < TAU_TAB_N) {
      ca = tau_tab<S>().ra[i];  // 0 at i = 3
      cb = tau_tab<S>().rb[i];
      cc = tau_tab<S>().rc[i];
    } else {
      ca = (i == 3) ? (S)0.0 : (S)0.25 / ((di - (S)2.0) * (di - (S)1.0));
      cb = (S)-0.5 / ((di - (S)2.0) * di);
      cc = (S)0.25 / ((di - (S)1.0) * di);
    }
    const S e2 = (i <= n - 4) ? tau_e(i - 2, lam) : (S)0.0;
#pragma unroll
    for (int q = 0; q < M; ++q) {
      S r = (S)0.0;
      if (fp[q] != nullptr && i - 3 - SB_PF_ROWS >= 0) pf_l2(fp[q] + (size_t)(i - 3 - SB_PF_ROWS) * fs[q]);
      if ((HOOK || fp[q] != nullptr) && WIN) {
        S fnew;  // f(i-3)
        if constexpr (HOOK) {
          fnew = (S)fh[q];
        } else if constexpr (EARLY) {
          fnew = (S)fpre[q];
          if (i >= 4) fpre[q] = fp[q][(size_t)(i - 4) * fs[q]];
        } else {
          fnew = (S)fp[q][(size_t)(i - 3) * fs[q]];
        }
        const S fm = (S)(pr ? wlo1[q] : wlo0[q]);          // f(i-1)
        const S fpl = (S)(pr ? whi1[q] : whi0[q]);         // f(i+1)
        if (i == 3) {
          r = (S)0.25 * fnew + fpl / (S)24.0 - fm / (S)6.0;
        } else {
          r = ca * fnew;
          if (i <= n - 2) r += cb * fm;
          if (i <= n - 4) r += cc * fpl;
        }
        if (pr) {
          whi1[q] = (FS)fm;
          wlo1[q] = (FS)fnew;
        } else {
          whi0[q] = (FS)fm;
          wlo0[q] = (FS)fnew;
        }
      } else if (fp[q] != nullptr) {
        const FS* __restrict__ F = fp[q];
        const size_t st = fs[q];
        if (i == 3) {
          r = (S)0.25 * (S)F[0] + (S)F[4 * st] / (S)24.0 - (S)F[2 * st] / (S)6.0;
        } else {
          r = ca * (S)F[(size_t)(i - 3) * st];
          if (i <= n - 2) r += cb * (S)F[(size_t)(i - 1) * st];
          if (i <= n - 4) r += cc * (S)F[(size_t)(i + 1) * st];
        }
      }
      if (i <= n - 4)
        r = (r - xb[q] * e2) * dinv;
      else if (i <= n - 2)
        r = r * dinv;
      xp[q][(size_t)(i - 1) * xs[q]] = r;
      if (FAST) {
        if (i <= n - 2) {
          if (i & 1)
            bs_odd[q] = bs_odd[q] + r * wnew;
          else
            bs_even[q] = bs_even[q] + r * wnew;
        }
      }
      xb[q] = xa[q];
      xa[q] = r;
    }
    q2 = q1;
    q1 = cnew;
    w2 = w1;
    w1 = wnew;
  }
  // c'(n-3), c'(n-2) are the unscaled c (d = 1 in the truncated rows)
  if (!CPC) {
    cpp[(size_t)(n - 4) * cs] = tau_c(n - 3, lam);
    cpp[(size_t)(n - 3) * cs] = tau_c(n - 2, lam);
  }
  if (FAST) {
    // after the sweep q1 = c'(1), q2 = c'(2), w1 = W(3), w2 = W(4)
    const S d1 = (S)1.0 / ((S)1.0 - q1 * w1);
    const S d2 = (S)1.0 / ((S)1.0 - q2 * w2);
#pragma unroll
    for (int q = 0; q < M; ++q) {
      S* __restrict__ X = xp[q];
      const size_t st = xs[q];
      // x(n), x(n-1): the sweep's first two rows, read back from the column
      // rather than held in registers through the sweep
      const S xn = X[(size_t)(n - 1) * st], xn1 = X[(size_t)(n - 2) * st];
      xa[q] = (bc1[q] - xn - bs_odd[q]) * d1;   // x(1)
      xb[q] = (bc2[q] - xn1 - bs_even[q]) * d2;  // x(2)
      X[0] = xa[q];
      X[st] = xb[q];
    }
    S ds0[M], ds1[M];
#pragma unroll
    for (int q = 0; q < M; ++q) {
      ds0[q] = xb[q];  // k = 1 (odd): 1^2 x_1
      ds1[q] = (S)0.0;
    }
    // row i's inputs are loaded during row i-1, before its stores (which
    // the compiler cannot move them past): the loads overlap a row's work
    S cn = cpp[0], xnx[M];
#pragma unroll
    for (int q = 0; q < M; ++q) xnx[q] = xp[q][2 * xs[q]];
#pragma unroll 4
    for (int i = 3; i <= n; ++i) {
      if (i - 1 + SB_PF_ROWS <= n - 1) pf_l2(cpp + (size_t)(i - 3 + SB_PF_ROWS) * cs);
      const S c = cn;
      S xc[M];
#pragma unroll
      for (int q = 0; q < M; ++q) xc[q] = xnx[q];
      if (i < n) {
        cn = cpp[(size_t)(i - 2) * cs];
#pragma unroll
        for (int q = 0; q < M; ++q) xnx[q] = xp[q][(size_t)i * xs[q]];
      }
      const S kk = (S)(i - 1) * (S)(i - 1);
#pragma unroll
      for (int q = 0; q < M; ++q) {
        const size_t o = (size_t)(i - 1) * xs[q];
        if (i - 1 + SB_PF_ROWS <= n - 1) pf_l2(xp[q] + o + (size_t)SB_PF_ROWS * xs[q]);
        const S v = xc[q] - c * xa[q];
        xp[q][o] = v;
        xa[q] = xb[q];
        xb[q] = v;
        if (i & 1)
          ds1[q] = ds1[q] + kk * v;  // k = i-1 even
        else
          ds0[q] = ds0[q] + kk * v;  // k odd
      }
    }
    if (dsum != nullptr) {
#pragma unroll
      for (int q = 0; q < M; ++q) {
        dsum[q][0] = ds0[q];
        dsum[q][1] = ds1[q];
      }
    }
    return;
  }
  const S d1 = (S)1.0 / ((S)1.0 - cpp[0] * wtp[2 * ws]);
  const S d2 = (S)1.0 / ((S)1.0 - cpp[cs] * wtp[3 * ws]);
#pragma unroll
  for (int q = 0; q < M; ++q) {
    S* __restrict__ X = xp[q];
    const size_t st = xs[q];
    S x1 = bc1[q] - X[(size_t)(n - 1) * st];
    S x2 = bc2[q] - X[(size_t)(n - 2) * st];
    for (int i = 5; i <= n - 2; i += 2) {
      x1 = x1 - X[(size_t)(i - 1) * st] * wtp[(size_t)(i - 1) * ws];
      x2 = x2 - X[(size_t)(i - 2) * st] * wtp[(size_t)(i - 2) * ws];
    }
    xa[q] = (x1 - X[2 * st] * wtp[2 * ws]) * d1;  // x(1)
    xb[q] = x2 * d2;                               // x(2)
    X[0] = xa[q];
    X[st] = xb[q];
  }
  // row i's inputs loaded during row i-1, as in the reordered variant
  S cn = cpp[0], xnx[M];
#pragma unroll
  for (int q = 0; q < M; ++q) xnx[q] = xp[q][2 * xs[q]];
#pragma unroll 4
  for (int i = 3; i <= n; ++i) {
    if (i - 1 + SB_PF_ROWS <= n - 1) pf_l2(cpp + (size_t)(i - 3 + SB_PF_ROWS) * cs);
    const S c = cn;
    S xc[M];
#pragma unroll
    for (int q = 0; q < M; ++q) xc[q] = xnx[q];
    if (i < n) {
      cn = cpp[(size_t)(i - 2) * cs];
#pragma unroll
      for (int q = 0; q < M; ++q) xnx[q] = xp[q][(size_t)i * xs[q]];
    }
#pragma unroll
    for (int q = 0; q < M; ++q) {
      const size_t o = (size_t)(i - 1) * xs[q];
      if (i - 1 + SB_PF_ROWS <= n - 1) pf_l2(xp[q] + o + (size_t)SB_PF_ROWS * xs[q]);
      const S v = xc[q] - c * xa[q];
      xp[q][o] = v;
      xa[q] = xb[q];
      xb[q] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Chebyshev transforms over pencils
// ---------------------------------------------------------------------------
// N > 0: the transform length 2(ny-1) is N, with the compile-time plan and
// NT threads per CTA; its first pass reads the columns (even extension
// folded into the index) and its last pass writes the n kept coefficients.
// SB_CHEB64_MINB: resident CTAs per SM the FP64 fixed-length variant's
// register budget is sized for (0: the compiler's choice, 56 registers at
// 256 threads; five CTAs, at 48 registers and a 16-byte spill, measured
// 0.82 -> 0.95 ms for the five-field inverse at 384x193x384)
#ifndef SB_CHEB64_MINB
#define SB_CHEB64_MINB 0
#endif
template <class T, int PB, class SI, class SO, int N = 0, int NT = 0>
__global__ void __launch_bounds__(NT > 0 ? NT : 256, (NT > 0 && sizeof(T) == 8) ? SB_CHEB64_MINB : 0)
    k_cheb(const typename C2<SI>::type* __restrict__ in, size_t in_fs, typename C2<SO>::type* __restrict__ out,
           size_t out_fs, Dims g, int inverse, double scale, FFTPlan plan, const typename C2<T>::type* __restrict__ tw,
           int skip_oddball) {
  typedef typename C2<T>::type V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n = g.nyp;
  const int Ny = n - 1;
  const int L = 2 * Ny;
  V* b0 = reinterpret_cast<V*>(smem_raw);
  V* b1 = b0 + (size_t)L * PB;
  const int f = blockIdx.y;
  const int p0 = g.p0 + blockIdx.x * PB;
  const typename C2<SI>::type* src = in + f * in_fs;
  typename C2<SO>::type* dst = out + f * out_fs;
  // row j (0..Ny) of pencil p0 + b, with the inverse transform's 1/2 on the
  // interior rows
  auto load = [&](int j, int b) -> V {
    const int p = p0 + b;
    double2 v = double2{0.0, 0.0};
    if (p < g.p1) {
      const auto q = src[(size_t)j * g.NP + p];
      v = double2{(double)q.x, (double)q.y};
    }
    if (inverse) {
      const double cb = (j == 0 || j == Ny) ? 1.0 : 0.5;
      v.x *= cb;
      v.y *= cb;
    }
    return V{(T)v.x, (T)v.y};
  };
  // coefficient k (0..Ny) of pencil p0 + b
  auto store = [&](int k, int b, V e) {
    const int p = p0 + b;
    if (p >= g.p1) return;
    if (skip_oddball && (p / g.nx2) == g.zodd) return;
    double fac = scale;
    if (!inverse) fac = scale / ((double)Ny * ((k == 0 || k == Ny) ? 2.0 : 1.0));
    dst[(size_t)k * g.NP + p] = typename C2<SO>::type{(SO)((double)e.x * fac), (SO)((double)e.y * fac)};
  };
  if constexpr (N > 0) {
    cfft_io<T, PB, N, -1, NT>([&](int m, int b) { return load(m <= Ny ? m : L - m, b); },
                              [&](int k, int b, V e) {
                                if (k <= Ny) store(k, b, e);
                              },
                              b0, b1, tw, threadIdx.x);
  } else {
    for (int t = threadIdx.x; t < n * PB; t += blockDim.x) {
      const int j = t / PB;
      const int b = t - j * PB;
      const V w = load(j, b);
      b0[j * PB + b] = w;
      if (j >= 1 && j <= Ny - 1) b0[(L - j) * PB + b] = w;
    }
    __syncthreads();
    V* res = fft_columns<T, PB>(b0, b1, plan, tw, -1);
    for (int t = threadIdx.x; t < n * PB; t += blockDim.x) {
      const int k = t / PB;
      store(k, t - k * PB, res[k * PB + (t - k * PB)]);
    }
  }
}

// ---------------------------------------------------------------------------
// per-pencil solve of one substep (all pencils except kx=kz=0 and the oddball)
// ---------------------------------------------------------------------------
struct PencilBufs {
  double2 *H1, *H2, *H3;          // Chebyshev nonlinear term (normalised)
  double2 *PV, *PW;               // state slots 6,7 (partial RHS, Chebyshev), updated in place
  double2 *HV, *HOM;              // forcing h_v, h_omega (storage FC), read by the last sweep
  double2 *PHI, *OM, *V, *DV;     // solutions phi, omega_y (storage SC), v; dv (FP64 path)
  double2 *OU, *OV, *OW, *OX, *OZ;  // outputs (Chebyshev)
  double *PHIH, *DVH;             // k_pencil_hom: phi_h, and D v_h for the FP64 path's sums
};

struct RKc {
  double an, bn, anp1, bnp1;
};

// Homogeneous solutions of one RK stage, cached: phi_h solves
// (D^2 - lam) phi_h = 0 with phi_h = 1 at both walls and v_h solves
// (D^2 - k^2) v_h = phi_h with v_h = 0 (linearbl.f:625-626, 1000-1001 with
// zero forcing).  They depend on k^2 and lam = k^2 + 2 Re/(a_n + b_n) only,
// so they are computed once per stage value of a_n + b_n (dt is fixed) with
// exactly the arithmetic of the per-substep solves (the same tau_solve
// column operations), and the pencil kernel reads v_h and the two parity
// sums of D v_h instead of solving for them every substep.
//   VHc: v_h, n x NP (row-major in y like the fields); HS[2p + s]: FAST: the
//   parity sums dsum of v_h; FP64 path: sum over j = s, s+2, ... of (D v_h)_j
//   in ascending order (the reference's order).
//   CF: the coefficient columns of both solves for this stage (c' and the
//   weights W of the lam solve, c' and W of the v solve; W only for the FP64
//   path), 4 x (n x NP), read back by k_pencil instead of being rewritten.
template <class SC, class FC>
__global__ void __launch_bounds__(128) k_pencil_hom(PencilBufs B, Dims g, const double* __restrict__ alfa,
                                                    const double* __restrict__ beta, double re, double anbn,
                                                    double* __restrict__ VHc, double* __restrict__ HS,
                                                    double* __restrict__ CF) {
  const int p = g.p0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.p1) return;
  const int kx = p % g.nx2;
  const int iz = p / g.nx2;
  if (iz == g.zodd || p == 0) return;
  const int n = g.nyp;
  const size_t NP = g.NP;
  const double a = alfa[kx], be = beta[iz];
  const double k2 = a * a + be * be;
  const double lam = k2 + 2.0 * re / anbn;
  constexpr bool FAST = !std::is_same<FC, double>::value;
  const ColT<SC> ph{reinterpret_cast<SC*>(B.PHIH) + p, NP};
  const size_t fr = (size_t)n * NP;
  {
    const ColT<FC> f[1] = {ColT<FC>{nullptr, 0}};
    const SC one[1] = {1};
    tau_solve<1, SC, FC, FAST>((SC)lam, n, f, &ph, one, one, ColT<SC>{reinterpret_cast<SC*>(CF) + p, NP},
                               ColT<SC>{reinterpret_cast<SC*>(CF + fr) + p, NP});
  }
  const Col vh{VHc + p, NP};
  double dsum[1][2] = {{0, 0}};
  const double b0[1] = {0};
  tau_solve<1, double, SC, FAST>(k2, n, &ph, &vh, b0, b0, Col{CF + 2 * fr + p, NP}, Col{CF + 3 * fr + p, NP}, dsum);
  if (FAST) {
    HS[2 * (size_t)p] = dsum[0][0];
    HS[2 * (size_t)p + 1] = dsum[0][1];
  } else {
    const Col dvh = col_r(B.DVH, p, NP);
    cheb_deriv(dvh, vh, n);
    for (int is = 0; is < 2; ++is) {
      double sh = 0.0;
      for (int j = is; j < n; j += 2) sh = sh + dvh[j];
      HS[2 * (size_t)p + is] = sh;
    }
  }
}

// IO: storage of the Chebyshev H inputs and of the u, v, w, omega_x, omega_z
// outputs (double2, or float2 under the mixed-precision path); all algebra
// and the other columns are FP64.
// SC: scalar of the omega_y / particular-phi Helmholtz solve; FC: storage of
// its forcing columns h_v, h_omega (read by the next partial RHS, never
// differentiated).  FP64 path: double/double; the mixed-precision path stores
// the forcing in float.  The fourth-order v solve, the superposition and every
// derivative are FP64 in both.  VHc, HS: this stage's homogeneous solution
// (k_pencil_hom).
// resident CTAs of 128 threads per SM the register budget is sized for
#ifndef SB_PENCIL_MINB
#define SB_PENCIL_MINB 4
#endif
template <class IO, class SC, class FC>
__global__ void __launch_bounds__(128, SB_PENCIL_MINB) k_pencil(PencilBufs B, Dims g, const double* __restrict__ alfa,
                                                const double* __restrict__ beta, double re, RKc rk,
                                                const double* __restrict__ VHc, const double* __restrict__ HS,
                                                double* __restrict__ CF) {
  typedef typename C2<SC>::type SC2;
  typedef typename C2<FC>::type FC2;
  const int p = g.p0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.p1) return;
  const int kx = p % g.nx2;
  const int iz = p / g.nx2;
  if (iz == g.zodd || p == 0) return;
  const int n = g.nyp;
  const size_t NP = g.NP;
  const double a = alfa[kx], be = beta[iz];
  const double k2 = a * a + be * be;
  const double k2i = 1.0 / k2;
  const double lam = k2 + 2.0 * re / (rk.an + rk.bn);
  const double c1 = 2.0 * re / (rk.an + rk.bn) * rk.an;
  // the mixed path (FP32 forcing columns) takes the reordered sums of
  // tau_solve<..., FAST>; the FP64 path keeps the reference's order
  constexpr bool FAST = !std::is_same<FC, double>::value;
  double dsum[2][2] = {{0, 0}, {0, 0}};
  // this pencil's column of each array; all arrays are distinct
#define COLP(name) double2* __restrict__ name = B.name + p
  COLP(PV); COLP(PW); COLP(V); COLP(DV);
#undef COLP
#define COLF(name) FC2* __restrict__ name = reinterpret_cast<FC2*>(B.name) + p
  COLF(HV); COLF(HOM);
#undef COLF
  SC2* __restrict__ OM = reinterpret_cast<SC2*>(B.OM) + p;
#define COLIO(name) IO* __restrict__ name = reinterpret_cast<IO*>(B.name) + p
  COLIO(H1); COLIO(H2); COLIO(H3); COLIO(OU); COLIO(OV); COLIO(OW); COLIO(OX); COLIO(OZ);
#undef COLIO
  const double* __restrict__ VH = VHc + p;

  // Nonlinear forcing of the omega_y and phi equations (linearbl.f:303-340),
  // one row per call in descending order: g = i alpha H1 + i beta H3 and its
  // y-derivative by the dcheb recurrence dg_j = dg_{j+2} + 2(j+1) g_{j+1}
  // (same operations as cheb_deriv), hv = -(dg + k^2 H2),
  // homy = i beta H1 - i alpha H3 (stored for the next partial RHS), and the
  // right-hand sides f_v = p_v - c1 hv, f_omega = p_omega - c1 homy returned
  // to the omega_y/phi solve, which consumes them in the same order: the
  // forcing never goes through memory.
  double2 g1 = double2{0.0, 0.0};                           // g_{j+1}
  double2 d1 = double2{0.0, 0.0}, d2 = double2{0.0, 0.0};  // dg_{j+1}, dg_{j+2}
  auto assemble = [&](int j, FC* fr) {
    const size_t o = j * NP;
    if (j >= SB_PF_ROWS) {
      const size_t op = o - (size_t)SB_PF_ROWS * NP;
      pf_l2(H1 + op); pf_l2(H2 + op); pf_l2(H3 + op); pf_l2(PV + op); pf_l2(PW + op);
    }
    const IO h1i = H1[o], h2i = H2[o], h3i = H3[o];
    const double2 h1 = {(double)h1i.x, (double)h1i.y}, h2 = {(double)h2i.x, (double)h2i.y};
    const double2 h3 = {(double)h3i.x, (double)h3i.y};
    const double2 pv = PV[o], pw = PW[o];
    double2 dg;
    if (j == n - 1) {
      dg = double2{0.0, 0.0};
    } else {
      const double f = 2.0 * (double)(j + 1);
      dg = (j == n - 2) ? double2{f * g1.x, f * g1.y} : double2{d2.x + f * g1.x, d2.y + f * g1.y};
    }
    d2 = d1;
    d1 = dg;
    if (j == 0) dg = double2{0.5 * dg.x, 0.5 * dg.y};
    g1 = double2{-a * h1.y - be * h3.y, a * h1.x + be * h3.x};
    const double2 hom = double2{-be * h1.y + a * h3.y, be * h1.x - a * h3.x};
    const FC2 homs = FC2{(FC)hom.x, (FC)hom.y};
    HOM[o] = homs;
    const double2 hv = double2{-(dg.x + k2 * h2.x), -(dg.y + k2 * h2.y)};
    const FC2 hvs = FC2{(FC)hv.x, (FC)hv.y};
    HV[o] = hvs;
    // f_v, f_omega rounded to the forcing storage type as when they were stored
    fr[0] = (FC)(pv.x - c1 * hv.x);
    fr[1] = (FC)(pv.y - c1 * hv.y);
    fr[2] = (FC)(pw.x - c1 * hom.x);
    fr[3] = (FC)(pw.y - c1 * hom.y);
  };
  // phi (particular) and omega_y: (D^2 - lam) psi = f  (linearbl.f:625-626)
  {
    auto cre = [&](double2* arr) { return ColT<SC>{reinterpret_cast<SC*>(arr) + 2 * (size_t)p, 2 * NP}; };
    auto cim = [&](double2* arr) { return ColT<SC>{reinterpret_cast<SC*>(arr) + 2 * (size_t)p + 1, 2 * NP}; };
    // rows n-1 and n-2 first; the solve asks for row i-3 at its row i
    FC fdummy[4];
    assemble(n - 1, fdummy);
    assemble(n - 2, fdummy);
    const ColT<FC> f[4] = {};
    const ColT<SC> x[4] = {cre(B.PHI), cim(B.PHI), cre(B.OM), cim(B.OM)};
    const SC bc0[4] = {0, 0, 0, 0};
    // coefficient columns of this stage from k_pencil_hom (same lam, same n)
    const size_t fr = (size_t)n * NP;
    tau_solve<4, SC, FC, FAST, true>((SC)lam, n, f, x, bc0, bc0, ColT<SC>{reinterpret_cast<SC*>(CF) + p, NP},
                                     ColT<SC>{reinterpret_cast<SC*>(CF + fr) + p, NP}, nullptr,
                                     [&](int i, FC* fo) { assemble(i - 3, fo); });
    // v from phi: (D^2 - k^2) v = phi  (linearbl.f:1000-1001), FP64
    const ColT<SC> fv[2] = {cre(B.PHI), cim(B.PHI)};
    const Col xv[2] = {col_re(B.V, p, NP), col_im(B.V, p, NP)};
    const double b0[2] = {0, 0};
    tau_solve<2, double, SC, FAST, true>(k2, n, fv, xv, b0, b0, Col{CF + 2 * fr + p, NP}, Col{CF + 3 * fr + p, NP},
                                         dsum);
  }
  const double hs0 = HS[2 * (size_t)p], hs1 = HS[2 * (size_t)p + 1];
  double cvr[2], cvi[2];
  if (FAST) {
    // parity sums of dv from v itself (returned by the v solve)
    const double hs[2] = {hs0, hs1};
    for (int is = 0; is < 2; ++is) {
      const double cinv = 1.0 / hs[is];
      cvr[1 - is] = (0.0 - dsum[0][is]) * cinv;
      cvi[1 - is] = (0.0 - dsum[1][is]) * cinv;
    }
  } else {
  // dv/dy = 0 at the walls: add the homogeneous solution per parity
  // (linearbl.f:1020-1085).  The parity sums of dv run in ascending order as
  // in the reference, so dv is stored by a backward derivative sweep.
  cheb_deriv(col_re(B.DV, p, NP), col_re(B.V, p, NP), n);
  cheb_deriv(col_im(B.DV, p, NP), col_im(B.V, p, NP), n);
  for (int is = 0; is < 2; ++is) {
    double sr = 0.0, si = 0.0;
    for (int j = is; j < n; j += 2) {
      const double2 dv = DV[j * NP];
      sr = sr + dv.x;
      si = si + dv.y;
    }
    const double cinv = 1.0 / (is == 0 ? hs0 : hs1);
    cvr[1 - is] = (0.0 - sr) * cinv;
    cvi[1 - is] = (0.0 - si) * cinv;
  }
  }
  // One backward sweep for everything after the superposition: the final v,
  // its first and second derivative, phi = D^2 v - k^2 v (tau, linearbl.f:
  // 1160-1170), D phi, D^2 phi, D omega_y, D^2 omega_y (chained dcheb
  // recurrences; each level's halving of coefficient 0 only touches its last
  // value), then u, w, omega_x, omega_z (loop 2800, :1193-1212) and the next
  // partial right-hand sides (:1696-1800).
  {
    const double c1n = 2.0 * re / (rk.anp1 + rk.bnp1);
    const double c2 = 2.0 * re * rk.bnp1 / (rk.anp1 + rk.bnp1);
    const double k2m = k2 - c1n;
    // value at j+1 and derivative values at j+1, j+2 of each chain
    double2 v1 = {0, 0}, dv1 = {0, 0}, dv2 = {0, 0}, ddv1 = {0, 0}, ddv2 = {0, 0};
    double2 ph1 = {0, 0}, dph1 = {0, 0}, dph2 = {0, 0}, ddph1 = {0, 0}, ddph2 = {0, 0};
    double2 om1 = {0, 0}, dom1 = {0, 0}, dom2 = {0, 0}, ddom1 = {0, 0}, ddom2 = {0, 0};
    auto step = [&](double2 x1, double2& b1, double2& b2, int j) -> double2 {
      // b_j from b_{j+2} = b2 and x_{j+1} = x1; updates (b1, b2) <- (b_j, b_{j+1})
      double2 b;
      if (j == n - 1) {
        b = double2{0.0, 0.0};
      } else {
        const double f = 2.0 * (double)(j + 1);
        b = (j == n - 2) ? double2{f * x1.x, f * x1.y} : double2{b2.x + f * x1.x, b2.y + f * x1.y};
      }
      b2 = b1;
      b1 = b;
      return (j == 0) ? double2{0.5 * b.x, 0.5 * b.y} : b;
    };
    for (int j = n - 1; j >= 0; --j) {
      const size_t o = j * NP;
      if (j >= SB_PF_ROWS) {
        const size_t op = o - (size_t)SB_PF_ROWS * NP;
        pf_l2(VH + op); pf_l2(V + op); pf_l2(OM + op); pf_l2(HV + op); pf_l2(HOM + op);
      }
      const double vh = VH[o];
      const double2 vp = V[o];
      const double2 v = double2{vp.x + cvr[j & 1] * vh, vp.y + cvi[j & 1] * vh};
      const SC2 omi = OM[o];
      const FC2 hvi = HV[o], homi = HOM[o];
      const double2 om = {(double)omi.x, (double)omi.y}, hv = {(double)hvi.x, (double)hvi.y};
      const double2 hom = {(double)homi.x, (double)homi.y};
      const double2 dv = step(v1, dv1, dv2, j);
      // second derivative from the first derivative at j+1 (before halving)
      const double2 ddv = step(dv2, ddv1, ddv2, j);
      const double2 phi = double2{ddv.x - k2 * v.x, ddv.y - k2 * v.y};
      const double2 dph = step(ph1, dph1, dph2, j);
      const double2 ddph = step(dph2, ddph1, ddph2, j);
      const double2 dom = step(om1, dom1, dom2, j);
      const double2 ddom = step(dom2, ddom1, ddom2, j);
      typedef decltype(IO::x) R;
      OU[o] = IO{(R)((-a * dv.y + be * om.y) * k2i), (R)((a * dv.x - be * om.x) * k2i)};
      OW[o] = IO{(R)((-a * om.y - be * dv.y) * k2i), (R)((a * om.x + be * dv.x) * k2i)};
      OZ[o] = IO{(R)((-be * dom.y + a * phi.y) * k2i), (R)((be * dom.x - a * phi.x) * k2i)};
      OX[o] = IO{(R)((-a * dom.y - be * phi.y) * k2i), (R)((a * dom.x + be * phi.x) * k2i)};
      OV[o] = IO{(R)v.x, (R)v.y};
      PV[o] = double2{-ddph.x + k2m * phi.x - c2 * hv.x, -ddph.y + k2m * phi.y - c2 * hv.y};
      PW[o] = double2{-ddom.x + k2m * om.x - c2 * hom.x, -ddom.y + k2m * om.y - c2 * hom.y};
      v1 = v;
      ph1 = phi;
      om1 = om;
    }
  }
}

// ---------------------------------------------------------------------------
// kx = kz = 0: mean flow with the constant-flux pressure gradient
// (linearbl.f:1214-1470 tau branch, ibc = 0; next partial RHS :1712-1733)
// One warp (lane 0 solves); FP64.  scratch: 12 columns of n doubles.
// ---------------------------------------------------------------------------
struct MeanArgs {
  double2 *H1, *H3;        // Chebyshev nonlinear term
  double *puw;             // [2][ny] partial RHS of the mean flow
  double *scal;            // [0] px, [1] mflux
  double *scr;             // scratch
  double2 *OU, *OV, *OW, *OX, *OZ, *PV, *PW;
  int cflux;
};

template <class IO>
__global__ void k_mean(MeanArgs A, Dims g, double re, RKc rk) {
  // One warp: the lanes move the columns between the state (strided by NP,
  // so a serial loop would wait one DRAM latency per row) and the contiguous
  // scratch columns; lane 0 does the solves in the reference's order.  The
  // scratch is global (L1-cached), not shared memory: this block runs beside
  // the pencil grid, whose SMs keep no shared-memory carveout, and a block
  // that needs shared memory would wait for the whole pencil wave to retire.
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  const int n = g.nyp;
  const int NP = g.NP;
  Col huw1{A.scr + 0 * n, 1}, huw2{A.scr + 1 * n, 1}, fu{A.scr + 2 * n, 1}, fw{A.scr + 3 * n, 1};
  Col U{A.scr + 4 * n, 1}, W{A.scr + 5 * n, 1}, DU{A.scr + 6 * n, 1}, DW{A.scr + 7 * n, 1};
  Col cp{A.scr + 8 * n, 1}, wt{A.scr + 9 * n, 1}, t1{A.scr + 10 * n, 1}, t2{A.scr + 11 * n, 1};
  const double c1 = 2.0 * re / (rk.an + rk.bn) * rk.an;
  for (int j = lane; j < n; j += 32) {
    huw1[j] = (double)reinterpret_cast<const IO*>(A.H1)[(size_t)j * NP].x;
    huw2[j] = (double)reinterpret_cast<const IO*>(A.H3)[(size_t)j * NP].x;
    fu[j] = A.puw[j] - c1 * huw1[j];
    fw[j] = A.puw[n + j] - c1 * huw2[j];
  }
  __syncwarp();
  if (lane == 0) {
    double px = A.scal[0];
    const double mflux = A.scal[1];
    fu[0] = fu[0] + 2.0 * re * px;
    const double lam = 0.0 + 2.0 * re / (rk.an + rk.bn);
    const double bz[1] = {0.0};
    {
      const Col f[2] = {fu, fw};
      const Col x[2] = {U, W};
      const double b0[2] = {0.0, 0.0};
      tau_solve<2>(lam, n, f, x, b0, b0, cp, wt);
    }
    if (A.cflux) {
      double m1 = 0.0;
      for (int j = 0; j < n; j += 2) m1 = m1 - U[j] * 2.0 / (double)(j * j - 1);
      fu[0] = fu[0] + 2.0 * re * px;
      tau_solve<1>(lam, n, &fu, &U, bz, bz, cp, wt);
      double m2 = 0.0;
      for (int j = 0; j < n; j += 2) m2 = m2 - U[j] * 2.0 / (double)(j * j - 1);
      fu[0] = fu[0] - 4.0 * re * px;
      px = px * (1.0 + (mflux - m1) / (m2 - m1));
      fu[0] = fu[0] + 2.0 * re * px;
      tau_solve<1>(lam, n, &fu, &U, bz, bz, cp, wt);
      A.scal[0] = px;
    }
    cheb_deriv(DU, U, n);
    cheb_deriv(DW, W, n);
    cheb_deriv(t1, DU, n);
    cheb_deriv(t2, DW, n);
  }
  __syncwarp();
  typedef decltype(IO::x) R;
  const double c1n = 2.0 * re / (rk.anp1 + rk.bnp1);
  const double c2 = 2.0 * re * rk.bnp1 / (rk.anp1 + rk.bnp1);
  for (int j = lane; j < n; j += 32) {
    reinterpret_cast<IO*>(A.OU)[(size_t)j * NP] = IO{(R)U[j], (R)0};
    reinterpret_cast<IO*>(A.OW)[(size_t)j * NP] = IO{(R)W[j], (R)0};
    reinterpret_cast<IO*>(A.OV)[(size_t)j * NP] = IO{(R)0, (R)0};
    reinterpret_cast<IO*>(A.OX)[(size_t)j * NP] = IO{(R)DW[j], (R)0};
    reinterpret_cast<IO*>(A.OZ)[(size_t)j * NP] = IO{(R)(-DU[j]), (R)0};
    A.PV[(size_t)j * NP] = double2{0.0, 0.0};
    A.PW[(size_t)j * NP] = double2{0.0, 0.0};
    A.puw[j] = -t1[j] - c1n * U[j] - c2 * huw1[j];
    A.puw[n + j] = -t2[j] - c1n * W[j] - c2 * huw2[j];
  }
}

// ---------------------------------------------------------------------------
// startup partial right-hand side and vorticities (bla/prhs.f), all pencils
// ---------------------------------------------------------------------------
struct PrhsBufs {
  double2 *U1, *U2, *U3;    // Chebyshev velocities
  double2 *OMY, *OX, *OZ, *PHI, *T1, *T2;
  double2 *PV, *PW;         // state slots 6,7
  double *puw;
};

static __global__ void k_prhs(PrhsBufs B, Dims g, const double* __restrict__ alfa, const double* __restrict__ beta,
                       double re, double an) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.NP) return;
  const int kx = p % g.nx2;
  const int iz = p / g.nx2;
  const int n = g.nyp;
  const int NP = g.NP;
  const double a = alfa[kx], be = beta[iz];
  const double k2 = a * a + be * be;
  const double lam = k2 - 2.0 * re / an;
  auto at = [&](double2* arr, int j) -> double2& { return arr[(size_t)j * NP + p]; };
  for (int j = 0; j < n; ++j) {
    const double2 u1 = at(B.U1, j), u3 = at(B.U3, j);
    at(B.OMY, j) = double2{-u1.y * be + u3.y * a, u1.x * be - u3.x * a};
  }
  cheb_deriv(col_re(B.T1, p, NP), col_re(B.U3, p, NP), n);
  cheb_deriv(col_im(B.T1, p, NP), col_im(B.U3, p, NP), n);
  for (int j = 0; j < n; ++j) {
    const double2 t = at(B.T1, j), u2 = at(B.U2, j);
    at(B.OX, j) = double2{t.x + u2.y * be, t.y - u2.x * be};
  }
  cheb_deriv(col_re(B.T1, p, NP), col_re(B.U1, p, NP), n);
  cheb_deriv(col_im(B.T1, p, NP), col_im(B.U1, p, NP), n);
  for (int j = 0; j < n; ++j) {
    const double2 t = at(B.T1, j), u2 = at(B.U2, j);
    at(B.OZ, j) = double2{-t.x - u2.y * a, -t.y + u2.x * a};
  }
  // phi = D^2 v - k^2 v
  cheb_deriv(col_re(B.T1, p, NP), col_re(B.U2, p, NP), n);
  cheb_deriv(col_im(B.T1, p, NP), col_im(B.U2, p, NP), n);
  cheb_deriv(col_re(B.T2, p, NP), col_re(B.T1, p, NP), n);
  cheb_deriv(col_im(B.T2, p, NP), col_im(B.T1, p, NP), n);
  for (int j = 0; j < n; ++j) {
    const double2 t = at(B.T2, j), u2 = at(B.U2, j);
    at(B.PHI, j) = double2{t.x - k2 * u2.x, t.y - k2 * u2.y};
  }
  // p_omega = -D^2 omega_y + lam omega_y
  cheb_deriv(col_re(B.T1, p, NP), col_re(B.OMY, p, NP), n);
  cheb_deriv(col_im(B.T1, p, NP), col_im(B.OMY, p, NP), n);
  cheb_deriv(col_re(B.T2, p, NP), col_re(B.T1, p, NP), n);
  cheb_deriv(col_im(B.T2, p, NP), col_im(B.T1, p, NP), n);
  for (int j = 0; j < n; ++j) {
    const double2 t = at(B.T2, j), om = at(B.OMY, j);
    at(B.PW, j) = double2{-t.x + lam * om.x, -t.y + lam * om.y};
  }
  // p_v = -D^2 phi + lam phi
  cheb_deriv(col_re(B.T1, p, NP), col_re(B.PHI, p, NP), n);
  cheb_deriv(col_im(B.T1, p, NP), col_im(B.PHI, p, NP), n);
  cheb_deriv(col_re(B.T2, p, NP), col_re(B.T1, p, NP), n);
  cheb_deriv(col_im(B.T2, p, NP), col_im(B.T1, p, NP), n);
  for (int j = 0; j < n; ++j) {
    const double2 t = at(B.T2, j), ph = at(B.PHI, j);
    at(B.PV, j) = double2{-t.x + lam * ph.x, -t.y + lam * ph.y};
  }
  if (p == 0) {
    // mean flow partial RHS: -2 Re/an U - D^2 U (prhs.f, zb = 1)
    cheb_deriv(col_re(B.T1, 0, NP), col_re(B.U1, 0, NP), n);
    cheb_deriv(col_re(B.T2, 0, NP), col_re(B.T1, 0, NP), n);
    for (int j = 0; j < n; ++j) B.puw[j] = -2.0 * re / an * at(B.U1, j).x - at(B.T2, j).x;
    cheb_deriv(col_re(B.T1, 0, NP), col_re(B.U3, 0, NP), n);
    cheb_deriv(col_re(B.T2, 0, NP), col_re(B.T1, 0, NP), n);
    for (int j = 0; j < n; ++j) B.puw[n + j] = -2.0 * re / an * at(B.U3, j).x - at(B.T2, j).x;
  }
}

}  // namespace sb
