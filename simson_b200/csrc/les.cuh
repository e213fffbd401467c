// ADM-RT large-eddy model on the device (iles = 1): the high-pass filtered
// velocities gu of the end of step 3 (bla/linearbl.f:1871-1960, and at start-up
// bla/prhs.f:95-193) and the relaxation term -chi gu added to H in step 2
// (bla/nonlinbl.f:920-965).  Filter tables: les_filter.h.
//
// One thread per (kx, kz) pencil and velocity component; the wall-normal
// filter is a five-point right-hand side and a pentadiagonal LU solve along the
// pencil, as the reference's hpf_y / lpf_y / pntdiag (bla/hpf_y.f,
// bla/lpf_y.f, bla/bandsolver.f): a forward sweep (right-hand side from a
// five-value register window, elimination) into a scratch column and a
// backward substitution out of it.  Pencils are columns of stride NP, so a
// warp reads 32 neighbouring complex values per row.
#pragma once
#include "fft.cuh"
#include "layout.cuh"

namespace sb {

// Per-row coefficients, LES_ROW doubles per row:
//   [0..4]  right-hand-side stencil of the high pass (g2 - g1)
//   [5..9]  right-hand-side stencil of the low pass (g1)
//   [10] e  [11] l1  [12] 1/d  [13] u1  [14] u2      (LU of the implicit A)
constexpr int LES_ROW = 15;

struct YFilter {
  const double* c;  // [nyp][LES_ROW]
  double fact2, factm2;
  int n;
};

template <class V>
SB_HD __forceinline__ double2 to_d2(V a) {
  return double2{(double)a.x, (double)a.y};
}

SB_HD __forceinline__ double2 axpy2(double a, double2 x, double2 y) { return double2{y.x + a * x.x, y.y + a * x.y}; }

// rs_j = sum_l b_l d_l, accumulated from l = 0 as the reference does
SB_HD __forceinline__ double2 stencil5(const double* b, const double2* w) {
  double2 s{0.0, 0.0};
#pragma unroll
  for (int l = 0; l < 5; ++l) {
    s.x = s.x + b[l] * w[l].x;
    s.y = s.y + b[l] * w[l].y;
  }
  return s;
}

// Applies the wall-normal filter to one complex column.
//   in(j)  : input value at row j (already scaled)
//   Z      : scratch column (stride zs)
//   put(j, x): receives the result at row j, j = n-1 down to 0
// hpf selects the high pass (zero at the walls) or the low pass (identity at
// the walls).
template <class In, class Put>
SB_HD __forceinline__ void yfilter_column(const YFilter& F, bool hpf, In in, double2* Z, size_t zs, Put put) {
  const int n = F.n;
  const int ob = hpf ? 0 : 5;
  auto C = [&](int j, int k) { return F.c[(size_t)j * LES_ROW + k]; };
  double2 w[5];
#pragma unroll
  for (int l = 0; l < 5; ++l) w[l] = in(l);
  // rows 0, 1, 2 (row 1 takes the row-2 combination that makes A pentadiagonal)
  const double2 r0 = hpf ? double2{0.0, 0.0} : w[0];
  const double2 r2 = stencil5(&F.c[2 * LES_ROW + ob], w);
  double2 r1 = stencil5(&F.c[1 * LES_ROW + ob], w);
  r1 = axpy2(F.fact2, r2, r1);
  double2 zm2, zm1, z;
  z = double2{r0.x * C(0, 12), r0.y * C(0, 12)};
  Z[0] = z;
  zm2 = z;
  z = double2{(r1.x - C(1, 11) * zm2.x) * C(1, 12), (r1.y - C(1, 11) * zm2.y) * C(1, 12)};
  Z[zs] = z;
  zm1 = z;
  z = double2{(r2.x - C(2, 10) * zm2.x - C(2, 11) * zm1.x) * C(2, 12),
              (r2.y - C(2, 10) * zm2.y - C(2, 11) * zm1.y) * C(2, 12)};
  Z[2 * zs] = z;
  zm2 = zm1;
  zm1 = z;
  double2 rprev = r2;
  for (int j = 3; j <= n - 3; ++j) {
#pragma unroll
    for (int l = 0; l < 4; ++l) w[l] = w[l + 1];
    w[4] = in(j + 2);
    const double2 r = stencil5(&F.c[(size_t)j * LES_ROW + ob], w);
    z = double2{(r.x - C(j, 10) * zm2.x - C(j, 11) * zm1.x) * C(j, 12),
                (r.y - C(j, 10) * zm2.y - C(j, 11) * zm1.y) * C(j, 12)};
    Z[(size_t)j * zs] = z;
    zm2 = zm1;
    zm1 = z;
    rprev = r;
  }
  {
    // row n-2 uses the last window d(n-5..n-1) and the row n-3 right-hand side
    const int j = n - 2;
    double2 r = stencil5(&F.c[(size_t)j * LES_ROW + ob], w);
    r = axpy2(F.factm2, rprev, r);
    z = double2{(r.x - C(j, 10) * zm2.x - C(j, 11) * zm1.x) * C(j, 12),
                (r.y - C(j, 10) * zm2.y - C(j, 11) * zm1.y) * C(j, 12)};
    Z[(size_t)j * zs] = z;
    zm2 = zm1;
    zm1 = z;
  }
  {
    const int j = n - 1;
    const double2 r = hpf ? double2{0.0, 0.0} : w[4];
    z = double2{(r.x - C(j, 10) * zm2.x - C(j, 11) * zm1.x) * C(j, 12),
                (r.y - C(j, 10) * zm2.y - C(j, 11) * zm1.y) * C(j, 12)};
  }
  // backward substitution
  double2 xp1 = z, xp2;
  put(n - 1, xp1);
  {
    const int j = n - 2;
    const double2 zj = Z[(size_t)j * zs];
    const double2 x = double2{zj.x - C(j, 13) * xp1.x, zj.y - C(j, 13) * xp1.y};
    put(j, x);
    xp2 = xp1;
    xp1 = x;
  }
  for (int j = n - 3; j >= 0; --j) {
    const double2 zj = Z[(size_t)j * zs];
    const double2 x = double2{zj.x - C(j, 13) * xp1.x - C(j, 14) * xp2.x, zj.y - C(j, 13) * xp1.y - C(j, 14) * xp2.y};
    put(j, x);
    xp2 = xp1;
    xp1 = x;
  }
}

// High-pass filtered velocity of one pencil column (component stored at
// src, stride s), written to gu (stride s); Z scratch.  mode = ihighorder.
template <class V>
SB_HD __forceinline__ void les_hpf_column(const YFilter& F, int mode, int iord, double lpf, double filt,
                                          const V* src, double2* gu, double2* Z, size_t s) {
  const int n = F.n;
  if (mode == 0) {
    for (int j = 0; j < n; ++j) {
      const double2 u = to_d2(src[(size_t)j * s]);
      gu[(size_t)j * s] = double2{u.x - lpf * u.x, u.y - lpf * u.y};
    }
    return;
  }
  if (mode == 1) {
    // gu = u; repeat: gu -= L_y (F_xz gu)
    for (int j = 0; j < n; ++j) gu[(size_t)j * s] = to_d2(src[(size_t)j * s]);
    for (int it = 0; it <= iord; ++it) {
      yfilter_column(
          F, false,
          [&](int j) {
            const double2 a = gu[(size_t)j * s];
            return double2{filt * a.x, filt * a.y};
          },
          Z, s,
          [&](int j, double2 x) {
            const double2 a = gu[(size_t)j * s];
            gu[(size_t)j * s] = double2{a.x - x.x, a.y - x.y};
          });
    }
    return;
  }
  // mode 2: H_y^(N+1) u, then gu = u - L_xz (u - H_y^(N+1) u)
  for (int it = 0; it <= iord; ++it) {
    if (it == 0)
      yfilter_column(
          F, true, [&](int j) { return to_d2(src[(size_t)j * s]); }, Z, s,
          [&](int j, double2 x) { gu[(size_t)j * s] = x; });
    else
      yfilter_column(
          F, true, [&](int j) { return gu[(size_t)j * s]; }, Z, s,
          [&](int j, double2 x) { gu[(size_t)j * s] = x; });
  }
  for (int j = 0; j < n; ++j) {
    const double2 u = to_d2(src[(size_t)j * s]);
    const double2 h = gu[(size_t)j * s];
    const double2 lo = double2{u.x - h.x, u.y - h.y};
    gu[(size_t)j * s] = double2{u.x - lpf * lo.x, u.y - lpf * lo.y};
  }
}

#ifdef __CUDACC__
// gu[ll] for ll = blockIdx.y (0..2) from the velocity slots of st (FP64 or
// FP32 storage); one thread per pencil.  skip_oddball leaves the kz = -nz/2
// plane alone (linearbl never visits it).
template <class V>
__global__ void __launch_bounds__(128) k_les_hpf(const V* __restrict__ st, double2* gu, double2* Z, YFilter F,
                                                 const double* __restrict__ lpf, const double* __restrict__ filt,
                                                 Dims g, int mode, int iord, int skip_oddball) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.NP) return;
  if (skip_oddball && p / g.nx2 == g.zodd) return;
  const size_t fld = (size_t)g.nyp * g.NP;
  const int ll = blockIdx.y;
  les_hpf_column(F, mode, iord, lpf[p], filt[p], st + ll * fld + p, gu + ll * fld + p, Z + ll * fld + p,
                 (size_t)g.NP);
}

// H_ll -= chi gu_ll nxp nzp on the stored modes, the oddball plane excepted
// (bla/nonlinbl.f:934-964: getxz returns zeros there).
template <class V>
__global__ void k_les_relax(V* __restrict__ h, const double2* __restrict__ gu, Dims g, double chi) {
  const size_t fld = (size_t)g.nyp * g.NP;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * fld) return;
  const int p = (int)(i % (size_t)g.NP);
  if (p / g.nx2 == g.zodd) return;
  const double2 q = gu[i];
  const double nxp = (double)g.nxp, nzp = (double)g.nzp;
  V a = h[i];
  a.x = a.x - chi * q.x * nxp * nzp;
  a.y = a.y - chi * q.y * nxp * nzp;
  h[i] = a;
}
#endif

}  // namespace sb
