// Pressure of the current velocity field: the reference's bla/nonlinp.f and
// bla/linearp.f, which bla/bla.f:2486-2527 runs after a step whose field is
// saved.  In the velocity-vorticity formulation the pressure is not carried;
// it solves
//   (D^2 - k^2) phi = i alpha H1 + D H2 + i beta H3,   p = phi - E,
// with H = u x (omega + 2 Omega) and 2E = |u|^2 formed on the dealiased grid
// as in step 2, and the Neumann conditions of the wall-normal momentum
// equation, D phi = H2 + (D^2 v - k^2 v)/Re - dv/dt at y = +-1
// (linearp.f:77-158).  The mean mode (kx = kz = 0) integrates H2 instead
// (linearp.f:172-186).
//
//   step-2 z-inverse (k_zinv) of u, v, w, omega
//   k_xpass_p    per z row: inverse x FFT, H1, H2, H3 and 2E (nonlinp.f:133-166),
//                forward x FFT, kept modes written over the row's own spectra
//   step-2 z-forward (k_zfwd) of H1, H2, H3 and 2E into scratch fields
//   k_press_div  i alpha H1 + i beta H3 (nonlinp.f:200-236)
//   Chebyshev transforms of that, H2 and E (k_cheb)
//   k_press      per pencil: the right-hand side, the Neumann data, the tau
//                solve of bla/crhsc.f, bla/setmac.f (neumann = 1) and
//                bla/tridc.f, the mean mode by bla/icheb.f, minus E
//   inverse Chebyshev transform of p (k_cheb)
// All FP64 (under FP32 state storage the FP32 fields are read and widened);
// the pencil arithmetic follows the reference's operation order.
#pragma once
#include "fft.cuh"
#include "layout.cuh"
#include "step2.cuh"
#include "step3.cuh"

namespace sb {

// One z row m of plane y per CTA: fields u+iv, w+i omega_x, omega_y+i omega_z
// of zb (z physical, x spectral), Hermitian-completed, inverse x FFT; H and
// 2E; forward x FFT of (H1 + i H2) and (H3 + i 2E); the kx < nx/2 spectra of
// H1, H2, H3, 2E written to fields 0..3 of the same row of zb (this CTA's own
// row: every read of it is done before the first barrier).
// fr: the fringe forcing of a spatial run, which the reference's pressure
// includes as well (bla/fringp.f, the forcing of bla/fring.f on H).
__global__ void __launch_bounds__(256) k_xpass_p(double2* __restrict__ zb, Dims g, FFTPlan plan,
                                                 const double2* __restrict__ tw, double rot, Fringe fr) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* bA = reinterpret_cast<double2*>(smem_raw);
  const int n = g.nxp;
  double2* bB = bA + (size_t)n * 3;
  const int m = blockIdx.x, y = blockIdx.y;
  const size_t fstride = (size_t)g.nyp * g.nzp * g.nx2;
  double2* row = zb + ((size_t)y * g.nzp + m) * g.nx2;
  for (int t = threadIdx.x; t < n * 3; t += blockDim.x) {
    const int k = t / 3, q = t - 3 * (t / 3);
    const double2* p0 = row + (size_t)(2 * q) * fstride;
    const double2* p1 = p0 + fstride;
    double2 z{0.0, 0.0};
    if (k == 0) {
      z = double2{p0[0].x, p1[0].x};
    } else if (k < g.nx2) {
      const double2 a = p0[k], b = p1[k];
      z = double2{a.x - b.y, a.y + b.x};
    } else if (k > n - g.nx2) {
      const int kk = n - k;
      const double2 a = p0[kk], b = p1[kk];
      z = double2{a.x + b.y, b.x - a.y};
    }
    bA[t] = z;
  }
  __syncthreads();
  double2* res = fft_columns<double, 3>(bA, bB, plan, tw, +1);
  double2* oth = (res == bA) ? bB : bA;
  const double r2 = 2.0 * rot;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double2 z0 = res[j * 3 + 0], z1 = res[j * 3 + 1], z2 = res[j * 3 + 2];
    const double u = z0.x, v = z0.y, w = z1.x, ox = z1.y, oy = z2.x, oz = z2.y;
    double h1 = v * (oz + r2) - w * oy;
    double h2 = w * ox - u * (oz + r2);
    double h3 = u * oy - v * ox;
    if (fr.lam != nullptr) fringe_apply<double>(fr, j, y, g.nyp, n, u, v, w, 0.0, 0.0, h1, h2, h3);
    const double e2 = u * u + v * v + w * w;
    oth[j * 2 + 0] = double2{h1, h2};
    oth[j * 2 + 1] = double2{h3, e2};
  }
  __syncthreads();
  double2* fres = fft_columns<double, 2>(oth, res, plan, tw, -1);
  for (int k = threadIdx.x; k < g.nx2; k += blockDim.x) {
    const int kk = (n - k) % n;
    const double2 a = fres[k * 2], b = fres[kk * 2];
    const double2 c = fres[k * 2 + 1], d = fres[kk * 2 + 1];
    row[k] = double2{(a.x + b.x) * 0.5, (a.y - b.y) * 0.5};
    row[fstride + k] = double2{(a.y + b.y) * 0.5, (b.x - a.x) * 0.5};
    row[2 * fstride + k] = double2{(c.x + d.x) * 0.5, (c.y - d.y) * 0.5};
    row[3 * fstride + k] = double2{(c.y + d.y) * 0.5, (d.x - c.x) * 0.5};
  }
}

// h[0] <- i alpha H1 + i beta H3 (h[0] = H1, h[2] = H3 on entry), every
// stored mode of every plane (nonlinp.f:200-236, stored as linearp reads it)
__global__ void k_press_div(double2* __restrict__ h, Dims g, const double* __restrict__ alfa,
                            const double* __restrict__ beta) {
  const size_t fld = (size_t)g.nyp * g.NP;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= fld) return;
  const int p = (int)(i % g.NP);
  const double a = alfa[p % g.nx2], b = beta[p / g.nx2];
  const double2 h1 = h[i], h3 = h[2 * fld + i];
  h[i] = double2{-a * h1.y - b * h3.y, a * h1.x + b * h3.x};
}

struct PressArgs {
  const double2 *CD, *CH2, *CE;  // Chebyshev coefficients: i alpha H1 + i beta H3, H2 (1/(nxp nzp)), E
  const double2 *PH2, *PE;       // physical H2 and 2E (walls, unnormalised)
  const double2* V;              // state slot 1 (v, physical y), FP64 storage
  const float2* Vf;              // the same under FP32 storage (V unused when set)
  double2* X;                    // right-hand side, then the Chebyshev coefficients of p
  double *Q, *Cc, *Dd, *Ee;      // real scratch columns [nyp][NP]
  const double* wd;              // [2][nyp]: second-derivative weights at y = +1 and y = -1
  const double *alfa, *beta;
  double re, c4t, cn, e2n;       // (1 - 1/it)/dt, 1/(nxp nzp), 2 nxp nzp
  int cim;
};

// bla/crhsc.f on one column F (0-based; n = ny): the tau rows of the
// Chebyshev right-hand side, the two boundary rows bc1, bc2 first.
__device__ __forceinline__ void press_crhsc(Col F, int n, double bc1, double bc2) {
  {
    const double tm1 = F[1];
    F[1] = F[2];
    F[2] = .25 * F[0] + F[4] / 24. - F[2] / 6.;
    F[0] = tm1;
  }
  for (int j = 4; j <= n - 4; j += 2) {
    const int y = j - 1, yy = j;
    const double rk1 = .25 / ((double)y * (double)(y - 1));
    const double rk2 = .5 / ((double)(y - 1) * (double)(y + 1));
    const double rk3 = .25 / ((double)y * (double)(y + 1));
    const double rk4 = .25 / ((double)yy * (double)(yy - 1));
    const double rk5 = .5 / ((double)(yy - 1) * (double)(yy + 1));
    const double rk6 = .25 / ((double)yy * (double)(yy + 1));
    const double tm1 = F[j - 1], tm2 = F[j];
    F[j - 1] = rk1 * F[0] + rk3 * F[j + 1] - rk2 * F[j - 1];
    F[j] = rk4 * F[1] + rk6 * F[j + 2] - rk5 * F[j];
    F[0] = tm1;
    F[1] = tm2;
  }
  const double tm1 = F[n - 4], tm2 = F[n - 3];
  {
    const int j = n - 4;
    F[n - 4] = .25 / ((double)j * (double)(j - 1)) * F[0] - .5 / ((double)(j - 1) * (double)(j + 1)) * F[n - 4];
  }
  {
    const int j = n - 3;
    F[n - 3] = .25 / ((double)j * (double)(j - 1)) * F[1] - .5 / ((double)(j - 1) * (double)(j + 1)) * F[n - 3];
  }
  F[n - 2] = .25 / ((double)(n - 2) * (double)(n - 3)) * tm1;
  F[n - 1] = .25 / ((double)(n - 1) * (double)(n - 2)) * tm2;
  F[0] = bc1;
  F[1] = bc2;
}

__device__ __forceinline__ double2 vload(const PressArgs& A, size_t i) {
  if (A.Vf) return double2{(double)A.Vf[i].x, (double)A.Vf[i].y};
  return A.V[i];
}

__global__ void __launch_bounds__(128) k_press(PressArgs A, Dims g) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= g.NP) return;
  const int iz = p / g.nx2;
  if (iz == g.zodd) return;  // linearp.f:64
  const int n = g.nyp;
  const size_t NP = g.NP;
  const double a = A.alfa[p % g.nx2], b = A.beta[iz];
  const double k2 = a * a + b * b;
  // Neumann data: H2 at the walls (linearp.f:77-88)
  double vr1 = A.PH2[p].x * A.cn, vi1 = A.PH2[p].y * A.cn;
  double vr2 = A.PH2[(size_t)(n - 1) * NP + p].x * A.cn, vi2 = A.PH2[(size_t)(n - 1) * NP + p].y * A.cn;
  // right-hand side D H2 + (i alpha H1 + i beta H3) (linearp.f:115-126)
  const Col Xr = col_re(A.X, p, (int)NP), Xi = col_im(A.X, p, (int)NP);
  cheb_deriv(Xr, col_re(const_cast<double2*>(A.CH2), p, (int)NP), n);
  cheb_deriv(Xi, col_im(const_cast<double2*>(A.CH2), p, (int)NP), n);
  for (int j = 0; j < n; ++j) {
    const double2 cd = A.CD[(size_t)j * NP + p];
    Xr[j] = Xr[j] + cd.x;
    Xi[j] = Xi[j] + cd.y;
  }
  // D^2 v at the walls from the quadrature weights, then the viscous and
  // time-derivative terms (linearp.f:130-150; v at the walls of the last
  // step is zero for the no-slip channel)
  double dr1 = 0., dr2 = 0., di1 = 0., di2 = 0.;
  for (int y = 0; y < n; ++y) {
    const double2 vv = vload(A, (size_t)y * NP + p);
    dr1 = dr1 + vv.x * A.wd[y];
    dr2 = dr2 + vv.x * A.wd[n + y];
    di1 = di1 + vv.y * A.wd[y];
    di2 = di2 + vv.y * A.wd[n + y];
  }
  const double2 v0 = vload(A, p), vn = vload(A, (size_t)(n - 1) * NP + p);
  vr1 = vr1 + (dr1 - k2 * v0.x) / A.re - (v0.x - 0.0) * A.c4t;
  vr2 = vr2 + (dr2 - k2 * vn.x) / A.re - (vn.x - 0.0) * A.c4t;
  vi1 = vi1 + (di1 - k2 * v0.y) / A.re - (v0.y - 0.0) * A.c4t;
  vi2 = vi2 + (di2 - k2 * vn.y) / A.re - (vn.y - 0.0) * A.c4t;
  press_crhsc(Xr, n, 0.5 * (vr1 - vr2), 0.5 * (vr1 + vr2));
  press_crhsc(Xi, n, 0.5 * (vi1 - vi2), 0.5 * (vi1 + vi2));
  // bla/setmac.f, neumann = 1: boundary rows q = k^2, tau rows c, d, e
  const Col Q{A.Q + p, NP}, C{A.Cc + p, NP}, D{A.Dd + p, NP}, E{A.Ee + p, NP};
  for (int i = 1; i <= n; ++i) Q[i - 1] = (double)(i - 1) * (double)(i - 1);
  for (int i = 1; i <= n - 6; ++i) {
    const int k = i + 1;
    const double rk1 = .25 / ((double)k * (double)(k - 1));
    const double rk2 = .5 / ((double)(k - 1) * (double)(k + 1));
    const double rk3 = .25 / ((double)k * (double)(k + 1));
    C[i - 1] = -rk1 * k2;
    D[i - 1] = 1. + rk2 * k2;
    E[i - 1] = -rk3 * k2;
  }
  C[0] = 2. * C[0];
  for (int i = n - 5; i <= n - 4; ++i) {
    const int k = i + 1;
    const double rk1 = .25 / ((double)k * (double)(k - 1));
    const double rk2 = .5 / ((double)(k - 1) * (double)(k + 1));
    C[i - 1] = -rk1 * k2;
    D[i - 1] = 1. + rk2 * k2;
    E[i - 1] = 0.;
  }
  for (int i = n - 3; i <= n - 2; ++i) {
    const int k = i + 1;
    const double rk1 = .25 / ((double)k * (double)(k - 1));
    C[i - 1] = -rk1 * k2;
    D[i - 1] = 1.;
    E[i - 1] = 0.;
  }
  // bla/tridc.f: elimination per parity, both right-hand sides in place
  for (int ns = 1; ns <= 2; ++ns) {
    const int nl = n - (n + ns) % 2;
    for (int i = nl - 2; i >= ns + 4; i -= 2) {
      D[i - 3] = 1. / D[i - 3];
      C[i - 3] = C[i - 3] * D[i - 3];
      D[i - 5] = D[i - 5] - C[i - 3] * E[i - 5];
      Xr[i - 1] = Xr[i - 1] * D[i - 3];
      Xr[i - 3] = Xr[i - 3] - Xr[i - 1] * E[i - 5];
      Xi[i - 1] = Xi[i - 1] * D[i - 3];
      Xi[i - 3] = Xi[i - 3] - Xi[i - 1] * E[i - 5];
    }
    D[ns - 1] = 1. / D[ns - 1];
    C[ns - 1] = C[ns - 1] * D[ns - 1];
    Xr[ns + 1] = Xr[ns + 1] * D[ns - 1];
    Xi[ns + 1] = Xi[ns + 1] * D[ns - 1];
    for (int i = nl; i >= ns + 2; i -= 2) Q[i - 3] = Q[i - 3] - C[i - 3] * Q[i - 1];
    for (int i = nl; i >= ns + 4; i -= 4) {
      Xr[ns - 1] = Xr[ns - 1] - Xr[i - 1] * Q[i - 1] - Xr[i - 3] * Q[i - 3];
      Xi[ns - 1] = Xi[ns - 1] - Xi[i - 1] * Q[i - 1] - Xi[i - 3] * Q[i - 3];
    }
    if ((nl - (ns + 2)) % 4 == 0) {
      Xr[ns - 1] = Xr[ns - 1] - Xr[ns + 1] * Q[ns + 1];
      Xi[ns - 1] = Xi[ns - 1] - Xi[ns + 1] * Q[ns + 1];
    }
    if (fabs(Q[ns - 1]) == 0.) {
      Xr[ns - 1] = 0.;
      Xi[ns - 1] = 0.;
    } else {
      Xr[ns - 1] = Xr[ns - 1] / Q[ns - 1];
      Xi[ns - 1] = Xi[ns - 1] / Q[ns - 1];
    }
    for (int i = ns + 2; i <= nl; i += 2) {
      Xr[i - 1] = Xr[i - 1] - C[i - 3] * Xr[i - 3];
      Xi[i - 1] = Xi[i - 1] - C[i - 3] * Xi[i - 3];
    }
  }
  if (p == 0) {
    // mean mode: the integral of H2 (linearp.f:172-186, bla/icheb.f), the
    // constant from E at y = -1
    const Col T = col_re(const_cast<double2*>(A.CH2), 0, (int)NP);
    const double bc0 = A.PE[(size_t)(n - 1) * NP].x / A.e2n;
    const double tn = A.cim ? T[n - 1] : 0.0;  // temp(ny) = 0 without cim
    auto tv = [&](int j) { return j == n - 1 ? tn : T[j]; };
    for (int i = 3; i <= n - 1; ++i) Xr[i - 1] = (tv(i - 2) - tv(i)) * (.5 / (double)(i - 1));
    Xr[n - 1] = tv(n - 2) * (.5 / (double)(n - 1));
    Xr[1] = tv(0) - tv(2) * .5;
    Xr[0] = bc0;
    for (int y = 2; y <= n - 1; y += 2) Xr[0] = Xr[0] + Xr[y - 1] - Xr[y];
    for (int j = 0; j < n; ++j) Xi[j] = 0.0;
  }
  // p = phi - E (linearp.f:188-193)
  for (int j = 0; j < n; ++j) {
    const double2 ce = A.CE[(size_t)j * NP + p];
    Xr[j] = Xr[j] - ce.x;
    Xi[j] = Xi[j] - ce.y;
  }
}

}  // namespace sb
