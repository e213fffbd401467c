// Step 3 with one warp per (kx, kz) pencil: the same algebra as k_pencil
// (bla/linearbl.f:257-1860 for the channel, ibc = 0, tau method), with every
// column of the pencil held in registers across the warp instead of being
// swept serially by one thread through memory.
//
// Rows: lane l holds the Chebyshev coefficients j = R l .. R l + R - 1
// (R even, R >= 2, 32 R >= ny), so H, p_v, p_omega are read once and the five
// outputs and the new p_v, p_omega written once; nothing else goes through
// memory.
//
//   * Chebyshev derivative (bla/dcheb.f): the closed form of its recurrence,
//     b_j = sum over k > j with k - j odd of 2 k a_k (b_0 halved), as suffix
//     sums: per lane by parity, a warp scan of the lane sums, then each lane
//     down its rows.
//   * Tau solve of (D^2 - lam) x = f (the system bla/setmacrhs.f and
//     bla/trid.f:120-200 eliminate; tau_solve in step3.cuh): rows 3..n couple
//     x_{i-2}, x_i, x_{i+2} and the two boundary rows sum the even and the
//     odd coefficients, so each parity class is a tridiagonal system bordered
//     by one full row.  With the class's first unknown y_0 as a parameter,
//     y = P + y_0 Q (P the rows with y_0 = 0, Q their response to y_0 = 1),
//     and y_0 = (b - sum P) / (1 + sum Q).  The tridiagonal rows are solved
//     by the partition method: each lane eliminates its own rows (Thomas)
//     leaving its last unknown; those 32 unknowns form a tridiagonal system
//     solved by parallel cyclic reduction over the lanes; each lane then
//     back-substitutes.  The systems are diagonally dominant
//     (|d| = 1 + |c| + |e| for lam >= 0), so neither stage needs pivoting.
//   * The homogeneous solutions phi_h, v_h of the wall-condition
//     superposition are extra columns of the same two solves (no per-stage
//     cache), and the parity sums of D v are warp reductions.
//
// The summation orders differ from the reference's serial recurrences
// (round-off level); the mixed-precision path uses this kernel.
#pragma once
#include "step3.cuh"

namespace sb {

constexpr unsigned WFULL = 0xffffffffu;

__device__ __forceinline__ double wshd(double v, int d) { return __shfl_down_sync(WFULL, v, d); }
__device__ __forceinline__ double wshu(double v, int d) { return __shfl_up_sync(WFULL, v, d); }
__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(WFULL, v, m);
  return v;
}

// b = D a for one complex column (R rows per lane); rows j >= n are ignored
// on input and undefined on output.
template <int R>
__device__ __forceinline__ void wderiv(const double2 (&a)[R], double2 (&b)[R], int lane, int n) {
  double se_x = 0.0, se_y = 0.0, so_x = 0.0, so_y = 0.0;  // sums of 2 k a_k over this lane's rows
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int k = R * lane + r;
    if (k < n) {
      const double f = 2.0 * (double)k;
      if (k & 1) {
        so_x += f * a[r].x;
        so_y += f * a[r].y;
      } else {
        se_x += f * a[r].x;
        se_y += f * a[r].y;
      }
    }
  }
  // inclusive suffix sums over the lanes, then the exclusive one (lanes above)
  double ex = se_x, ey = se_y, ox = so_x, oy = so_y;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double t0 = wshd(ex, d), t1 = wshd(ey, d), t2 = wshd(ox, d), t3 = wshd(oy, d);
    if (lane + d < 32) {
      ex += t0;
      ey += t1;
      ox += t2;
      oy += t3;
    }
  }
  double Se_x = wshd(ex, 1), Se_y = wshd(ey, 1), So_x = wshd(ox, 1), So_y = wshd(oy, 1);
  if (lane == 31) Se_x = Se_y = So_x = So_y = 0.0;
#pragma unroll
  for (int r = R - 1; r >= 0; --r) {
    const int j = R * lane + r;
    double bx = (j & 1) ? Se_x : So_x, by = (j & 1) ? Se_y : So_y;  // k > j of the other parity
    if (j == 0) {
      bx *= 0.5;
      by *= 0.5;
    }
    b[r] = double2{bx, by};
    if (j < n) {
      const double f = 2.0 * (double)j;
      if (j & 1) {
        So_x += f * a[r].x;
        So_y += f * a[r].y;
      } else {
        Se_x += f * a[r].x;
        Se_y += f * a[r].y;
      }
    }
  }
}

// Tau-system row of Chebyshev coefficient j >= 2 (1-based row i = j + 1):
// c x_{j-2} + d x_j + e x_{j+2} = rhs (tau_c/d/e of bla/setmacrhs.f with the
// truncation of the last rows, as tau_solve eliminates them).
// The lam-independent factors come from the global table (each lane reads
// its own rows; rows beyond it are computed).
__device__ __forceinline__ void wtau_row(int j, int n, double lam, double& c, double& d, double& e) {
  const int i = j + 1;
  const int m = i - 2;
  if (m >= 1 && m < TAU_TAB_N) {
    c = __ldg(&kTauGlobal.c[m]) * lam;
    d = (i <= n - 2) ? 1.0 + __ldg(&kTauGlobal.d[m]) * lam : 1.0;
    e = (i <= n - 4) ? __ldg(&kTauGlobal.e[m]) * lam : 0.0;
    return;
  }
  c = tau_c(m, lam);
  d = (i <= n - 2) ? tau_d(m, lam) : 1.0;
  e = (i <= n - 4) ? tau_e(m, lam) : 0.0;
}

// Solves (D^2 - lam) x_q = f_q, q < NC, with the boundary rows
// sum_{k even} x_k = bc1[q], sum_{k odd} x_k = bc2[q] (x(+-1) = bc1 +- bc2).
// f and x may be the same array.  Rows j >= n of x are set to 0.
template <int R, int NC>
__device__ __forceinline__ void wtau(double lam, int n, double (&w)[NC + 1][R], const double (&bc1)[NC],
                                     const double (&bc2)[NC], int lane) {
  static_assert(R % 2 == 0, "an even number of rows per lane keeps the parity of row r equal to r's");
  constexpr int NQ = NC + 1;  // columns plus the response Q to the class's first unknown
  // ---- right-hand sides rows j >= 2: f(j-2), f(j), f(j+2) with halos of two
  // rows from each neighbouring lane
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    const double lo1 = wshu(w[q][R - 2], 1), lo0 = wshu(w[q][R - 1], 1);  // rows R l - 2, R l - 1
    const double hi0 = wshd(w[q][0], 1), hi1 = wshd(w[q][1], 1);          // rows R l + R, R l + R + 1
    double fr[R + 4];
    fr[0] = lo1;
    fr[1] = lo0;
#pragma unroll
    for (int r = 0; r < R; ++r) fr[r + 2] = w[q][r];
    fr[R + 2] = hi0;
    fr[R + 3] = hi1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = R * lane + r;
      const int i = j + 1;
      double v = 0.0;
      if (j >= 2 && j < n) {
        const double fm2 = fr[r], f0 = fr[r + 2], fp2 = fr[r + 4];
        if (i == 3) {
          v = 0.25 * fm2 + fp2 / 24.0 - f0 / 6.0;
        } else if (i < TAU_TAB_N) {
          v = __ldg(&kTauGlobal.ra[i]) * fm2;
          if (i <= n - 2) v += __ldg(&kTauGlobal.rb[i]) * f0;
          if (i <= n - 4) v += __ldg(&kTauGlobal.rc[i]) * fp2;
        } else {
          const double di = (double)i;
          v = (0.25 / ((di - 2.0) * (di - 1.0))) * fm2;
          if (i <= n - 2) v += (-0.5 / ((di - 2.0) * di)) * f0;
          if (i <= n - 4) v += (0.25 / ((di - 1.0) * di)) * fp2;
        }
      }
      w[q][r] = v;
    }
  }
  // response to the class's first unknown (rows 0 and 1): -c in rows 2, 3
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = R * lane + r;
    double c, d, e;
    wtau_row(j, n, lam, c, d, e);
    w[NC][r] = (j == 2 || j == 3) ? -c : 0.0;
  }
  // ---- this lane's rows of each class (j >= 2, j < n) are consecutive in
  // steps of two rows; the last one is the separator, the others are
  // eliminated (Thomas) in terms of the previous lane's separator zp and this
  // lane's z: x = u + L zp + U z (u in w, L, U per row)
  int cnt[2] = {0, 0}, last[2] = {-1, -1}, first[2] = {-1, -1};
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = R * lane + r;
    if (j >= 2 && j < n) {
      const int s = r & 1;
      if (first[s] < 0) first[s] = r;
      last[s] = r;
      cnt[s]++;
    }
  }
  double dp[R], L[R], U[R];
  // forward elimination over the interior rows (ascending); the interior
  // row before row r of the same class is r - 2
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = R * lane + r;
    dp[r] = 1.0;
    L[r] = 0.0;
    U[r] = 0.0;
    const int s = r & 1;
    if (j < 2 || j >= n || r == last[s]) continue;
    double c, d, e;
    wtau_row(j, n, lam, c, d, e);
    if (j == 2 || j == 3) c = 0.0;  // the first unknown is carried by Q
    if (r < 2 || r - 2 < first[s]) {
      dp[r] = d;
      L[r] = -c;
    } else if (r >= 2) {
      double cm, dm, em;
      wtau_row(j - 2, n, lam, cm, dm, em);
      const double wgt = c / dp[r >= 2 ? r - 2 : 0];
      dp[r] = d - wgt * em;
      L[r] = -wgt * L[r >= 2 ? r - 2 : 0];
#pragma unroll
      for (int q = 0; q < NQ; ++q) w[q][r] -= wgt * w[q][r >= 2 ? r - 2 : 0];
    }
  }
  // backward substitution over the interior rows (descending)
#pragma unroll
  for (int r = R - 1; r >= 0; --r) {
    const int j = R * lane + r;
    const int s = r & 1;
    if (j < 2 || j >= n || r == last[s]) continue;
    double c, d, e;
    wtau_row(j, n, lam, c, d, e);
    const double inv = 1.0 / dp[r];
    if (r + 2 >= R || r + 2 == last[s]) {
      // the last interior row couples to this lane's separator z
      U[r] = -e * inv;
      L[r] *= inv;
#pragma unroll
      for (int q = 0; q < NQ; ++q) w[q][r] *= inv;
    } else {
      const int rn = r + 2 < R ? r + 2 : r;
      U[r] = (0.0 - e * U[rn]) * inv;
      L[r] = (L[r] - e * L[rn]) * inv;
#pragma unroll
      for (int q = 0; q < NQ; ++q) w[q][r] = (w[q][r] - e * w[q][rn]) * inv;
    }
  }
  // ---- reduced system, one unknown (the separator) per lane and class:
  // A z_{l-1} + B z_l + C z_{l+1} = D
  double A[2], Bc[2], C[2], D[2][NQ];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    // first row of this lane's class s, for the lane below: (m, u, L, U)
    double fu[NQ], fl = 0.0, fU = 0.0;
    const int fr0 = first[s];
#pragma unroll
    for (int q = 0; q < NQ; ++q) fu[q] = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (r == fr0) {
        fl = L[r];
        fU = U[r];
#pragma unroll
        for (int q = 0; q < NQ; ++q) fu[q] = w[q][r];
      }
    const double mnext = wshd((double)cnt[s], 1);
    const double lnext = wshd(fl, 1), unext = wshd(fU, 1);
    double unx[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) unx[q] = wshd(fu[q], 1);
    const bool has_next = lane < 31 && mnext > 0.5;
    A[s] = 0.0;
    Bc[s] = 1.0;
    C[s] = 0.0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) D[s][q] = 0.0;
    if (cnt[s] == 0) continue;
    const int rs = last[s];
    const int j = R * lane + rs;
    double c, d, e;
    wtau_row(j, n, lam, c, d, e);
    if (j == 2 || j == 3) c = 0.0;
    double rhs[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      rhs[q] = 0.0;
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (r == rs) rhs[q] = w[q][r];
    }
    if (cnt[s] >= 2) {
      // the interior row two below the separator
      const int rp = rs - 2;
      double lp = 0.0, upp = 0.0, uq[NQ];
#pragma unroll
      for (int q = 0; q < NQ; ++q) uq[q] = 0.0;
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (r == rp) {
          lp = L[r];
          upp = U[r];
#pragma unroll
          for (int q = 0; q < NQ; ++q) uq[q] = w[q][r];
        }
      A[s] = c * lp;
      Bc[s] = d + c * upp;
#pragma unroll
      for (int q = 0; q < NQ; ++q) D[s][q] = rhs[q] - c * uq[q];
    } else {
      A[s] = c;
      Bc[s] = d;
#pragma unroll
      for (int q = 0; q < NQ; ++q) D[s][q] = rhs[q];
    }
    if (has_next && e != 0.0) {
      if (mnext > 1.5) {
        Bc[s] += e * lnext;
        C[s] = e * unext;
#pragma unroll
        for (int q = 0; q < NQ; ++q) D[s][q] -= e * unx[q];
      } else {
        C[s] = e;
      }
    }
  }
  // ---- parallel cyclic reduction over the lanes (both classes)
#pragma unroll
  for (int dd = 1; dd < 32; dd <<= 1) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double Am = wshu(A[s], dd), Bm = wshu(Bc[s], dd), Cm = wshu(C[s], dd);
      const double Ap = wshd(A[s], dd), Bp = wshd(Bc[s], dd), Cp = wshd(C[s], dd);
      const double k1 = (lane >= dd) ? A[s] / Bm : 0.0;
      const double k2 = (lane + dd < 32) ? C[s] / Bp : 0.0;
      A[s] = (lane >= dd) ? -k1 * Am : 0.0;
      C[s] = (lane + dd < 32) ? -k2 * Cp : 0.0;
      Bc[s] = Bc[s] - k1 * Cm - k2 * Ap;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const double Dm = wshu(D[s][q], dd), Dp = wshd(D[s][q], dd);
        D[s][q] = D[s][q] - k1 * Dm - k2 * Dp;
      }
    }
  }
  // ---- back substitution, then y_0 from the boundary row
  double ps[2][NQ];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    double z[NQ], zp[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      z[q] = D[s][q] / Bc[s];
      zp[q] = wshu(z[q], 1);
      if (lane == 0) zp[q] = 0.0;
      ps[s][q] = 0.0;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = R * lane + r;
      if (j < 2 || j >= n || (r & 1) != s) continue;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const double v = (r == last[s]) ? z[q] : w[q][r] + L[r] * zp[q] + U[r] * z[q];
        w[q][r] = v;
        ps[s][q] += v;
      }
    }
#pragma unroll
    for (int q = 0; q < NQ; ++q) ps[s][q] = wsum(ps[s][q]);
  }
#pragma unroll
  for (int s = 0; s < 2; ++s) {
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      const double b = s == 0 ? bc1[q] : bc2[q];
      const double y0 = (b - ps[s][q]) / (1.0 + ps[s][NC]);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = R * lane + r;
        if ((r & 1) != s) continue;
        if (j >= n)
          w[q][r] = 0.0;
        else if (j < 2)
          w[q][r] = y0;
        else
          w[q][r] += y0 * w[NC][r];
      }
    }
  }
}

// One warp per pencil of this context's range (kx = kz = 0 and the oddball
// plane excluded).  IO: storage of H and of the outputs (float2 on the
// mixed path); FC: rounding of the forcing columns h_v, h_omega and of the
// right-hand sides (float on the mixed path, as k_pencil stores them).
// SB_PWARP_MINB4/8: resident CTAs per SM the register budget is sized for,
// by rows per lane (0: the compiler's choice).  R = 4 (ny <= 127): four CTAs
// at 128 registers (a 64-byte spill) keep every pencil of the 64x97x64 LES
// grid resident at once, where the compiler's 166-174 registers left two or
// three: its step 0.648 -> 0.553 ms (FP64), 0.487 -> 0.401 ms (mixed).
#ifndef SB_PWARP_MINB4
#define SB_PWARP_MINB4 4
#endif
#ifndef SB_PWARP_MINB8
#define SB_PWARP_MINB8 0
#endif
template <class IO, class FC, int R>
__global__ void __launch_bounds__(128, R <= 4 ? SB_PWARP_MINB4 : SB_PWARP_MINB8)
    k_pencil_w(PencilBufs B, Dims g, const double* __restrict__ alfa,
                                                  const double* __restrict__ beta, double re, RKc rk) {
  const int lane = threadIdx.x & 31;
  const int p = g.p0 + (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  if (p >= g.p1) return;
  const int kx = p % g.nx2;
  const int iz = p / g.nx2;
  if (iz == g.zodd || p == 0) return;  // the whole warp leaves together
  const int n = g.nyp;
  const size_t NP = g.NP;
  const double a = alfa[kx], be = beta[iz];
  const double k2 = a * a + be * be;
  const double k2i = 1.0 / k2;
  const double lam = k2 + 2.0 * re / (rk.an + rk.bn);
  const double c1 = 2.0 * re / (rk.an + rk.bn) * rk.an;
  const IO* __restrict__ H1 = reinterpret_cast<const IO*>(B.H1) + p;
  const IO* __restrict__ H2 = reinterpret_cast<const IO*>(B.H2) + p;
  const IO* __restrict__ H3 = reinterpret_cast<const IO*>(B.H3) + p;
  double2* __restrict__ PV = B.PV + p;
  double2* __restrict__ PW = B.PW + p;

  // ---- forcing (linearbl.f:303-340): g = i alpha H1 + i beta H3, dg = D g,
  // h_v = -(dg + k^2 H2), h_omega = i beta H1 - i alpha H3, and the
  // right-hand sides f_v = p_v - c1 h_v, f_omega = p_omega - c1 h_omega
  double2 gg[R], dg[R];
  FC hvx[R], hvy[R], hmx[R], hmy[R];
  double wl[6][R];  // f_v re, im, f_omega re, im, phi_h's zero forcing, and the solve's Q column
  {
    double2 h2[R], pv[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = R * lane + r;
      double2 h1 = {0.0, 0.0}, h3 = {0.0, 0.0}, pw = {0.0, 0.0};
      h2[r] = double2{0.0, 0.0};
      pv[r] = double2{0.0, 0.0};
      if (j < n) {
        const IO x1 = H1[(size_t)j * NP], x2 = H2[(size_t)j * NP], x3 = H3[(size_t)j * NP];
        h1 = double2{(double)x1.x, (double)x1.y};
        h2[r] = double2{(double)x2.x, (double)x2.y};
        h3 = double2{(double)x3.x, (double)x3.y};
        pv[r] = PV[(size_t)j * NP];
        pw = PW[(size_t)j * NP];
      }
      gg[r] = double2{-a * h1.y - be * h3.y, a * h1.x + be * h3.x};
      const double2 hom = double2{-be * h1.y + a * h3.y, be * h1.x - a * h3.x};
      hmx[r] = (FC)hom.x;
      hmy[r] = (FC)hom.y;
      // right-hand sides rounded to the forcing storage type, as k_pencil does
      wl[2][r] = (double)(FC)(pw.x - c1 * hom.x);
      wl[3][r] = (double)(FC)(pw.y - c1 * hom.y);
      wl[4][r] = 0.0;
      wl[5][r] = 0.0;
    }
    wderiv<R>(gg, dg, lane, n);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double2 hv = double2{-(dg[r].x + k2 * h2[r].x), -(dg[r].y + k2 * h2[r].y)};
      hvx[r] = (FC)hv.x;
      hvy[r] = (FC)hv.y;
      wl[0][r] = (double)(FC)(pv[r].x - c1 * hv.x);
      wl[1][r] = (double)(FC)(pv[r].y - c1 * hv.y);
    }
  }
  // ---- phi (particular), omega_y and phi_h: (D^2 - lam) psi = f
  // (linearbl.f:625-626); phi_h has zero forcing and the wall values 1
  {
    const double bc[5] = {0.0, 0.0, 0.0, 0.0, 1.0};
    wtau<R, 5>(lam, n, wl, bc, bc, lane);
  }
  // wl: phi_p re, im, omega re, im, phi_h
  // ---- v from phi: (D^2 - k^2) v = phi (linearbl.f:1000-1001), for the
  // particular phi and for phi_h (v_h)
  double vv[4][R];  // v_p re, im, v_h, Q
#pragma unroll
  for (int r = 0; r < R; ++r) {
    vv[0][r] = wl[0][r];
    vv[1][r] = wl[1][r];
    vv[2][r] = wl[4][r];
    vv[3][r] = 0.0;
  }
  {
    const double bc[3] = {0.0, 0.0, 0.0};
    wtau<R, 3>(k2, n, vv, bc, bc, lane);
  }
  // ---- dv/dy = 0 at the walls (linearbl.f:1020-1085): the parity sums of
  // D v, sum_{j even} (D x)_j = sum_{k odd} k^2 x_k and sum_{j odd} (D x)_j =
  // sum_{k even} k^2 x_k, of v_p and v_h fix the amount of v_h per parity
  double s_r[2] = {0.0, 0.0}, s_i[2] = {0.0, 0.0}, s_h[2] = {0.0, 0.0};
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int k = R * lane + r;
    if (k >= n) continue;
    const double kk = (double)k * (double)k;
    const int is = (k & 1) ? 0 : 1;  // odd k -> the sum over even j
    s_r[is] += kk * vv[0][r];
    s_i[is] += kk * vv[1][r];
    s_h[is] += kk * vv[2][r];
  }
  double cvr[2], cvi[2];
#pragma unroll
  for (int is = 0; is < 2; ++is) {
    const double sr = wsum(s_r[is]), si = wsum(s_i[is]), sh = wsum(s_h[is]);
    const double cinv = 1.0 / sh;
    cvr[1 - is] = (0.0 - sr) * cinv;
    cvi[1 - is] = (0.0 - si) * cinv;
  }
  // ---- the final v, its derivatives, phi = D^2 v - k^2 v (tau,
  // linearbl.f:1160-1170), D phi, D^2 phi, D omega_y, D^2 omega_y; u, w,
  // omega_x, omega_z (loop 2800, :1193-1212) and the next partial right-hand
  // sides (:1696-1800)
  double2 v[R], om[R], t1[R], t2[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = R * lane + r;
    const double vh = vv[2][r];
    v[r] = double2{vv[0][r] + cvr[j & 1] * vh, vv[1][r] + cvi[j & 1] * vh};
    om[r] = double2{wl[2][r], wl[3][r]};
  }
  typedef decltype(IO::x) RT;
  IO* __restrict__ OU = reinterpret_cast<IO*>(B.OU) + p;
  IO* __restrict__ OV = reinterpret_cast<IO*>(B.OV) + p;
  IO* __restrict__ OW = reinterpret_cast<IO*>(B.OW) + p;
  IO* __restrict__ OX = reinterpret_cast<IO*>(B.OX) + p;
  IO* __restrict__ OZ = reinterpret_cast<IO*>(B.OZ) + p;
  const double c1n = 2.0 * re / (rk.anp1 + rk.bnp1);
  const double c2 = 2.0 * re * rk.bnp1 / (rk.anp1 + rk.bnp1);
  const double k2m = k2 - c1n;
  // dv -> t1; u, w need dv and omega
  wderiv<R>(v, t1, lane, n);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = R * lane + r;
    if (j >= n) continue;
    const size_t o = (size_t)j * NP;
    const double2 dv = t1[r], w_ = om[r];
    OU[o] = IO{(RT)((-a * dv.y + be * w_.y) * k2i), (RT)((a * dv.x - be * w_.x) * k2i)};
    OW[o] = IO{(RT)((-a * w_.y - be * dv.y) * k2i), (RT)((a * w_.x + be * dv.x) * k2i)};
    OV[o] = IO{(RT)v[r].x, (RT)v[r].y};
  }
  // phi = D^2 v - k^2 v (into v), then D phi, D^2 phi
  wderiv<R>(t1, t2, lane, n);
#pragma unroll
  for (int r = 0; r < R; ++r) v[r] = double2{t2[r].x - k2 * v[r].x, t2[r].y - k2 * v[r].y};
  wderiv<R>(v, t1, lane, n);
  wderiv<R>(t1, t2, lane, n);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = R * lane + r;
    if (j >= n) continue;
    const double2 phi = v[r], ddph = t2[r];
    PV[(size_t)j * NP] = double2{-ddph.x + k2m * phi.x - c2 * (double)hvx[r], -ddph.y + k2m * phi.y - c2 * (double)hvy[r]};
  }
  // D omega_y -> t1 (omega_x, omega_z need it with phi), D^2 omega_y -> t2
  wderiv<R>(om, t1, lane, n);
  wderiv<R>(t1, t2, lane, n);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = R * lane + r;
    if (j >= n) continue;
    const size_t o = (size_t)j * NP;
    const double2 dom = t1[r], phi = v[r], ddom = t2[r], w_ = om[r];
    OZ[o] = IO{(RT)((-be * dom.y + a * phi.y) * k2i), (RT)((be * dom.x - a * phi.x) * k2i)};
    OX[o] = IO{(RT)((-a * dom.y - be * phi.y) * k2i), (RT)((a * dom.x + be * phi.x) * k2i)};
    PW[o] = double2{-ddom.x + k2m * w_.x - c2 * (double)hmx[r], -ddom.y + k2m * w_.y - c2 * (double)hmy[r]};
  }
}

// Rows per lane for ny: even (a row's parity is then its slot's, known at
// compile time), at least two (the boundary rows 0 and 1 stay in lane 0),
// 32 R >= ny; 0 when ny is beyond the instantiated range.
inline int pencil_warp_rows(int ny) {
  const int r = 2 * ((ny + 63) / 64);
  return r <= 8 ? r : 0;
}

template <class IO, class FC>
bool launch_pencil_warp(cudaStream_t s, const PencilBufs& B, const Dims& g, const double* alfa, const double* beta,
                        double re, RKc rk) {
  const long long threads = 32LL * (g.p1 - g.p0);
  const unsigned blocks = (unsigned)((threads + 127) / 128);
  switch (pencil_warp_rows(g.nyp)) {
#define SB_PW_CASE(RR) \
  case RR:             \
    k_pencil_w<IO, FC, RR><<<blocks, 128, 0, s>>>(B, g, alfa, beta, re, rk); \
    return true;
    SB_PW_CASE(2) SB_PW_CASE(4) SB_PW_CASE(6) SB_PW_CASE(8)
#undef SB_PW_CASE
    default:
      return false;
  }
}

// kx = kz = 0 with one warp (the algebra of k_mean, linearbl.f:1214-1470 tau
// branch, ibc = 0, and the next partial right-hand side :1712-1733): U and W
// from (D^2 - lam) U = f_u, (D^2 - lam) W = f_w with lam = 2 Re/(a_n + b_n).
// Under constant flux the reference solves for U three times (px, 2 px, the
// corrected px); the system being linear, the warp solves once for f_u, f_w
// and the unit forcing G of row 0 and forms the same three solutions as
// U + s G.  Rows as in k_pencil_w (R per lane).
template <class IO, int R>
__global__ void __launch_bounds__(32) k_mean_w(MeanArgs A, Dims g, double re, RKc rk) {
  const int lane = threadIdx.x & 31;
  if (blockIdx.x != 0 || threadIdx.x >= 32) return;
  const int n = g.nyp;
  const size_t NP = g.NP;
  const double c1 = 2.0 * re / (rk.an + rk.bn) * rk.an;
  const double lam = 0.0 + 2.0 * re / (rk.an + rk.bn);
  double w[4][R];  // f_u, f_w, unit forcing of row 0; Q
  double h1[R], h3[R];
  double px = A.scal[0];
  const double mflux = A.scal[1];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = R * lane + r;
    h1[r] = h3[r] = 0.0;
    w[0][r] = w[1][r] = w[2][r] = w[3][r] = 0.0;
    if (j < n) {
      h1[r] = (double)reinterpret_cast<const IO*>(A.H1)[(size_t)j * NP].x;
      h3[r] = (double)reinterpret_cast<const IO*>(A.H3)[(size_t)j * NP].x;
      w[0][r] = A.puw[j] - c1 * h1[r];
      w[1][r] = A.puw[n + j] - c1 * h3[r];
      if (j == 0) {
        w[0][r] = w[0][r] + 2.0 * re * px;
        w[2][r] = 1.0;
      }
    }
  }
  {
    const double b0[3] = {0.0, 0.0, 0.0};
    wtau<R, 3>(lam, n, w, b0, b0, lane);
  }
  if (A.cflux) {
    // flux m = sum over even j of -U_j 2/(j^2 - 1) of U and of G
    double mu = 0.0, mg = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int j = R * lane + r;
      if (j < n && !(j & 1)) {
        const double wj = -2.0 / (double)(j * j - 1);
        mu += w[0][r] * wj;
        mg += w[2][r] * wj;
      }
    }
    mu = wsum(mu);
    mg = wsum(mg);
    const double m1 = mu, m2 = mu + 2.0 * re * px * mg;  // U, then U with 2 Re px more in row 0
    const double pxn = px * (1.0 + (mflux - m1) / (m2 - m1));
    const double sft = 2.0 * re * (pxn - px);
#pragma unroll
    for (int r = 0; r < R; ++r) w[0][r] += sft * w[2][r];
    px = pxn;
    if (lane == 0) A.scal[0] = px;
  }
  double2 uw[R], d1[R], d2[R];
#pragma unroll
  for (int r = 0; r < R; ++r) uw[r] = double2{w[0][r], w[1][r]};
  wderiv<R>(uw, d1, lane, n);
  wderiv<R>(d1, d2, lane, n);
  typedef decltype(IO::x) RT;
  const double c1n = 2.0 * re / (rk.anp1 + rk.bnp1);
  const double c2 = 2.0 * re * rk.bnp1 / (rk.anp1 + rk.bnp1);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = R * lane + r;
    if (j >= n) continue;
    const size_t o = (size_t)j * NP;
    reinterpret_cast<IO*>(A.OU)[o] = IO{(RT)uw[r].x, (RT)0};
    reinterpret_cast<IO*>(A.OW)[o] = IO{(RT)uw[r].y, (RT)0};
    reinterpret_cast<IO*>(A.OV)[o] = IO{(RT)0, (RT)0};
    reinterpret_cast<IO*>(A.OX)[o] = IO{(RT)d1[r].y, (RT)0};
    reinterpret_cast<IO*>(A.OZ)[o] = IO{(RT)(-d1[r].x), (RT)0};
    A.PV[o] = double2{0.0, 0.0};
    A.PW[o] = double2{0.0, 0.0};
    A.puw[j] = -d2[r].x - c1n * uw[r].x - c2 * h1[r];
    A.puw[n + j] = -d2[r].y - c1n * uw[r].y - c2 * h3[r];
  }
}

template <class IO>
bool launch_mean_warp(cudaStream_t s, const MeanArgs& M, const Dims& g, double re, RKc rk) {
  switch (pencil_warp_rows(g.nyp)) {
#define SB_MW_CASE(RR) \
  case RR:             \
    k_mean_w<IO, RR><<<1, 32, 0, s>>>(M, g, re, rk); \
    return true;
    SB_MW_CASE(2) SB_MW_CASE(4) SB_MW_CASE(6) SB_MW_CASE(8)
#undef SB_MW_CASE
    default:
      return false;
  }
}

}  // namespace sb
