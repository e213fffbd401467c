// Plane statistics of the state (the reference's bla/boxamp.f, evaluated by
// nonlinbl at the start of a full step when iamp > 0): per y-plane sums over
// the stored Fourier modes, kx > 0 counted twice for their -kx partners
// (Parseval), the kx = kz = 0 mode and the oddball kz = -nz/2 left out:
//   amp(y,1..3) <u'^2>, <v'^2>, <w'^2>      amp(y,4..6) <omega'_i^2>
//   amp(y,7)   <|omega_y|^2 / k^2>          amp(y,8)    <u'v'>
//   amp(y,9..12) mean U, W, Omega_x, Omega_z (the kx = kz = 0 mode)
//   amp(y,13) not written by boxamp (zero here)
//   amp(y,14..18) <u'w'>, <v'w'>, <u'u'>, <v'v'>, <w'w'>
//   amp(y,19..20) zero
// Sums run over the modes of the coarse grid (kx = 0..nx/2-1, kz = -nz/2+1 ..
// nz/2-1) exactly as bla/boxamp.f:55-240 does; omega_y = i beta u - i alpha w
// is formed from u and w.  One CTA per plane; FP64 accumulation whatever the
// storage type.  Output layout amp[k][y] (Fortran amp(nyp,20)).
#pragma once
#include "fft.cuh"
#include "layout.cuh"

namespace sb {

template <class S>
__global__ void __launch_bounds__(256) k_amp(const typename C2<S>::type* __restrict__ st, Dims g,
                                             const double* __restrict__ alfa, const double* __restrict__ beta,
                                             double* __restrict__ amp) {
  constexpr int NS = 13;
  const int y = blockIdx.x;
  const size_t slot = (size_t)g.nyp * g.NP;
  const size_t base = (size_t)y * g.NP;
  double acc[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) acc[k] = 0.0;
  for (int p = threadIdx.x; p < g.NP; p += blockDim.x) {
    const int kx = p % g.nx2, iz = p / g.nx2;
    if ((kx == 0 && iz == 0) || iz == g.zodd) continue;
    const double wgt = (kx > 0) ? 2.0 : 1.0;
    const auto u = st[base + p], v = st[slot + base + p], w = st[2 * slot + base + p];
    const auto ox = st[3 * slot + base + p], oz = st[4 * slot + base + p];
    const double a = alfa[kx], be = beta[iz];
    const double ur = u.x, ui = u.y, vr = v.x, vi = v.y, wr = w.x, wi = w.y;
    const double oxr = ox.x, oxi = ox.y, ozr = oz.x, ozi = oz.y;
    const double oyr = -be * ui + a * wi, oyi = be * ur - a * wr;
    const double uu = ur * ur + ui * ui, vv = vr * vr + vi * vi, ww = wr * wr + wi * wi;
    const double oy2 = oyr * oyr + oyi * oyi;
    acc[0] += uu * wgt;
    acc[1] += vv * wgt;
    acc[2] += ww * wgt;
    acc[3] += (oxr * oxr + oxi * oxi) * wgt;
    acc[4] += oy2 * wgt;
    acc[5] += (ozr * ozr + ozi * ozi) * wgt;
    acc[6] += oy2 / (a * a + be * be) * wgt;
    acc[7] += (ur * vr + ui * vi) * wgt;
    acc[8] += (ur * wr + ui * wi) * wgt;
    acc[9] += (vr * wr + vi * wi) * wgt;
    acc[10] += uu * wgt;
    acc[11] += vv * wgt;
    acc[12] += ww * wgt;
  }
  __shared__ double red[8][NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    double v = acc[k];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < NS) {
    double s = 0.0;
    for (int wv = 0; wv < (int)(blockDim.x >> 5); ++wv) s += red[wv][threadIdx.x];
    const int k = threadIdx.x;
    const int col = (k < 8) ? k : k + 5;  // amp(y,1..8) <- k 0..7, amp(y,14..18) <- k 8..12
    amp[(size_t)col * g.nyp + y] = s;
  }
  if (threadIdx.x == 0) {
    amp[(size_t)8 * g.nyp + y] = (double)st[base].x;              // amp(y,9)  U
    amp[(size_t)9 * g.nyp + y] = (double)st[2 * slot + base].x;   // amp(y,10) W
    amp[(size_t)10 * g.nyp + y] = (double)st[3 * slot + base].x;  // amp(y,11) Omega_x
    amp[(size_t)11 * g.nyp + y] = (double)st[4 * slot + base].x;  // amp(y,12) Omega_z
    amp[(size_t)12 * g.nyp + y] = 0.0;
    amp[(size_t)18 * g.nyp + y] = 0.0;
    amp[(size_t)19 * g.nyp + y] = 0.0;
  }
}

}  // namespace sb
