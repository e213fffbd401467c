// xy statistics of the velocity field on the device: the reference's
// bla/boxxys.f, which bla/bla.f:2069-2107 runs on every xz-plane at the start
// of a step that takes a sample (weight dtn, then sumw += dtn).  Per sample
// u, v, w, omega_x, omega_z, omega_y and the nine gradients du_i/dx_j go to
// physical space on the nx x nz grid, and the z averages of the one-point
// moments, times dtn, are added to xys(x, y, s) (boxxys.f:562-1380):
//    1-3  u_i              4-6  u_i^2            7-9  omega_i
//   10-12 omega_i^2       13-15 uv, uw, vw
//   25-27 sum_j (du_i/dx_j)^2                    28-30 sum_j du_1j du_2j, du_1j du_3j, du_2j du_3j
//   43-44 running min / max over z of u - <u>_z
//   45    S_ij S_ij       46-51 S_11, S_12, S_13, S_22, S_23, S_33
//   63-65 u_i^3           66-72 u^2 v, u^2 w, v^2 u, v^2 w, w^2 u, w^2 v, u v w
//   75-77 u_i^4
// With the pressure of the sampled state at hand (sgpu_pressure since the
// last change of the state, as the reference requires a pressure computed
// at the end of the previous step, bla/bla.f:1833-1840), also
//   31 p   32 p^2   33-35 u_i p   36-38 p du_i/dx_i   39-42 p uy, p vz, p wx, p uz
//   73-74 p vx, p wy   78-79 p^3, p^4          (boxxys.f:895-990, 1343-1400)
// The LES (52-62, 80-82) and MHD (83-96) entries need fields this path does
// not carry and stay zero, as in the reference built without them; 16-24
// are never written by the reference.
//
//   k_xys_zinv    per plane and kx block: the 15 spectral fields
//                 (boxxys.f:246-350: omega_y from u and w, the y derivatives
//                 from the vorticity and continuity), inverse z FFT.  The
//                 kz = -nz/2 mode is zero in every field (getxz.f:58-63 clears
//                 it on the unpadded grid).
//   k_xys_acc     per plane and group of z rows: inverse x FFT (two real rows
//                 per complex transform), the moments of each point
//                 accumulated in registers by the thread that owns its x;
//                 the group's sums and the physical u rows written out
//   k_xys_add     per (y, x): the groups' sums added to xys in group order
//   k_xys_minmax  per (y, x): <u>_z in z order, then the running min / max
//                 of u - <u>_z (boxxys.f:991-1035)
//
// FP64 arithmetic whatever the state storage.  Device layout of xys:
// [s][y][x] (the reference's xys(x, y, s) with leading dimensions nx, nyp).
#pragma once
#include "fft.cuh"
#include "layout.cuh"
#include "les_dyn.cuh"

namespace sb {

constexpr int XYS_NF = 16;     // spectral fields: u v w, omega x y z, du_ij (i-major), p
constexpr int XYS_NC = 8;      // complex x transforms carrying the 16 real rows
constexpr int XYS_NACC = 41;   // accumulated velocity entries (all but 43-44)
constexpr int XYS_NACC_P = 57;  // with the pressure entries
constexpr int XYS_NS = 96;     // entries of the reference's xys (bla/par.f nxys)
constexpr int XYS_GROUPS = 8;  // z-row groups per plane in k_xys_acc

// reference entry (1-based) of accumulator k
__device__ __host__ constexpr int xys_entry(int k) {
  return k < 15 ? k + 1 : k < 21 ? k + 10 : k < 28 ? k + 24 : k < 38 ? k + 35 : k < 41 ? k + 37
       : k < 53 ? k - 10 : k == 53 ? 73 : k == 54 ? 74 : k == 55 ? 78 : 79;
}

template <class V>
__device__ __forceinline__ double2 xys_spec_field(const V* st, const double2* pr, size_t slot, size_t off, int f,
                                                  double a, double b) {
  auto ld = [&](int s) { const V q = st[(size_t)s * slot + off]; return double2{(double)q.x, (double)q.y}; };
  switch (f) {
    case 0: return ld(0);
    case 1: return ld(1);
    case 2: return ld(2);
    case 3: return ld(3);
    case 4: {
      // omega_y = i beta u - i alpha w (boxxys.f:246-251)
      const double2 u = ld(0), w = ld(2);
      return double2{-b * u.y + a * w.y, b * u.x - a * w.x};
    }
    case 5: return ld(4);
    case 15: return pr ? pr[off] : double2{0.0, 0.0};  // pressure (getxz of slot 8)
    default: return sgs_spec_field(st, slot, off, f - 6, a, b, 1);  // du_i/dx_j (boxxys.f:323-366)
  }
}

template <class V, int KB>
__global__ void k_xys_zinv(const V* __restrict__ st, const double2* __restrict__ pr, double2* __restrict__ spec,
                           SgsGrid G, FFTPlan plan, const double2* __restrict__ tw,
                           const double* __restrict__ alfa, const double* __restrict__ beta) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* b0 = reinterpret_cast<double2*>(smem_raw);
  double2* b1 = b0 + (size_t)G.nz * KB;
  const int y = blockIdx.y;
  const int kx0 = blockIdx.x * KB;
  const size_t slot = (size_t)G.nyp * G.NP;
  for (int f = 0; f < XYS_NF; ++f) {
    for (int t = threadIdx.x; t < G.nz * KB; t += blockDim.x) {
      const int iz = t / KB;
      const int kx = kx0 + t - iz * KB;
      double2 val{0.0, 0.0};
      if (kx < G.nx2 && iz != G.zodd)
        val = xys_spec_field(st, pr, slot, (size_t)y * G.NP + (size_t)iz * G.nx2 + kx, f, alfa[kx], beta[iz]);
      b0[t] = val;
    }
    __syncthreads();
    double2* res = fft_columns<double, KB>(b0, b1, plan, tw, +1);
    for (int t = threadIdx.x; t < G.nz * KB; t += blockDim.x) {
      const int m = t / KB;
      const int kx = kx0 + t - m * KB;
      if (kx < G.nx2) spec[(((size_t)f * G.nyp + y) * G.nz + m) * G.nx2 + kx] = res[t];
    }
    __syncthreads();
  }
}

// blockDim.x >= nx (nx <= MAXT <= 512); thread j owns x = j.  part: [XYS_GROUPS][XYS_NACC_P][nyp][nx];
// PRES: the pressure entries too (field 15 holds p).
// uphys: [nyp][nz][nx].  c = dtn / nz, the weight of one point
// (boxxys.f:556, nfzsym = 0).
// MAXT: the block size the register budget is sized for.  The accumulators
// stay in registers across the z rows: at 512 threads (128 registers) 512
// bytes of them spill (240 without the pressure entries), at 384 threads
// (168 registers, grids with nx <= 384) 160 bytes (16).
template <bool PRES, int MAXT = 512>
__global__ void __launch_bounds__(MAXT) k_xys_acc(const double2* __restrict__ spec, double* __restrict__ part,
                                                  double* __restrict__ uphys, SgsGrid G, FFTPlan plan,
                                                  const double2* __restrict__ tw, double c) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* bA = reinterpret_cast<double2*>(smem_raw);
  double2* bB = bA + (size_t)G.nx * XYS_NC;
  const int grp = blockIdx.x, y = blockIdx.y;
  const int n = G.nx;
  const int j = threadIdx.x;
  const size_t fs = (size_t)G.nyp * G.nz * G.nx2;
  const int m0 = (int)((long long)G.nz * grp / XYS_GROUPS), m1 = (int)((long long)G.nz * (grp + 1) / XYS_GROUPS);
  constexpr int NACC = PRES ? XYS_NACC_P : XYS_NACC;
  double acc[NACC];
#pragma unroll
  for (int k = 0; k < NACC; ++k) acc[k] = 0.0;
  for (int m = m0; m < m1; ++m) {
    const size_t row = ((size_t)y * G.nz + m) * G.nx2;
    for (int t = threadIdx.x; t < n * XYS_NC; t += blockDim.x) {
      const int k = t / XYS_NC, cc = t - XYS_NC * (t / XYS_NC);
      const double2* a = spec + (size_t)(2 * cc) * fs + row;
      const double2* b = (2 * cc + 1 < XYS_NF) ? spec + (size_t)(2 * cc + 1) * fs + row : nullptr;
      bA[k * XYS_NC + cc] = sgs_pair(a, b, k, n, G.nx2);
    }
    __syncthreads();
    const double2* res = fft_columns<double, XYS_NC>(bA, bB, plan, tw, +1);
    if (j < n) {
      double q[16];
#pragma unroll
      for (int cc = 0; cc < XYS_NC; ++cc) {
        const double2 z = res[j * XYS_NC + cc];
        q[2 * cc] = z.x;
        q[2 * cc + 1] = z.y;
      }
      const double u = q[0], v = q[1], w = q[2];
      const double* om = q + 3;
      const double* du = q + 6;  // du[3 i + j] = du_i / dx_j
      uphys[((size_t)y * G.nz + m) * n + j] = u;
      const double uu = u * u, vv = v * v, ww = w * w;
      acc[0] += u * c;
      acc[1] += v * c;
      acc[2] += w * c;
      acc[3] += uu * c;
      acc[4] += vv * c;
      acc[5] += ww * c;
      acc[6] += om[0] * c;
      acc[7] += om[1] * c;
      acc[8] += om[2] * c;
      acc[9] += om[0] * om[0] * c;
      acc[10] += om[1] * om[1] * c;
      acc[11] += om[2] * om[2] * c;
      acc[12] += u * v * c;
      acc[13] += u * w * c;
      acc[14] += v * w * c;
      // dissipation tensor re eps_ij = du_i/dx_k du_j/dx_k (boxxys.f:849-891)
#pragma unroll
      for (int i = 0; i < 3; ++i)
        acc[15 + i] += (du[3 * i] * du[3 * i] + du[3 * i + 1] * du[3 * i + 1] + du[3 * i + 2] * du[3 * i + 2]) * c;
      acc[18] += (du[0] * du[3] + du[1] * du[4] + du[2] * du[5]) * c;
      acc[19] += (du[0] * du[6] + du[1] * du[7] + du[2] * du[8]) * c;
      acc[20] += (du[3] * du[6] + du[4] * du[7] + du[5] * du[8]) * c;
      // strain rate (boxxys.f:1037-1090)
      const double s1 = du[0], s2 = .5 * (du[3] + du[1]), s3 = .5 * (du[6] + du[2]);
      const double s4 = du[4], s5 = .5 * (du[5] + du[7]), s6 = du[8];
      acc[21] += (s1 * s1 + s4 * s4 + s6 * s6 + 2. * (s2 * s2 + s3 * s3 + s5 * s5)) * c;
      acc[22] += s1 * c;
      acc[23] += s2 * c;
      acc[24] += s3 * c;
      acc[25] += s4 * c;
      acc[26] += s5 * c;
      acc[27] += s6 * c;
      // third and fourth moments (boxxys.f:1276-1380)
      acc[28] += uu * u * c;
      acc[29] += vv * v * c;
      acc[30] += ww * w * c;
      acc[31] += uu * v * c;
      acc[32] += uu * w * c;
      acc[33] += vv * u * c;
      acc[34] += vv * w * c;
      acc[35] += ww * u * c;
      acc[36] += ww * v * c;
      acc[37] += u * v * w * c;
      acc[38] += uu * uu * c;
      acc[39] += vv * vv * c;
      acc[40] += ww * ww * c;
      if constexpr (PRES) {
        const double p = q[15];
        acc[41] += p * c;
        acc[42] += p * p * c;
        acc[43] += u * p * c;
        acc[44] += v * p * c;
        acc[45] += w * p * c;
        acc[46] += p * du[0] * c;  // p ux
        acc[47] += p * du[4] * c;  // p vy
        acc[48] += p * du[8] * c;  // p wz
        acc[49] += p * du[1] * c;  // p uy
        acc[50] += p * du[5] * c;  // p vz
        acc[51] += p * du[6] * c;  // p wx
        acc[52] += p * du[2] * c;  // p uz
        acc[53] += p * du[3] * c;  // p vx
        acc[54] += p * du[7] * c;  // p wy
        acc[55] += p * p * p * c;
        acc[56] += p * p * (p * p) * c;
      }
    }
    __syncthreads();
  }
  if (j < n) {
    const size_t plane = (size_t)G.nyp * n;
#pragma unroll
    for (int k = 0; k < NACC; ++k)
      part[((size_t)grp * XYS_NACC_P + k) * plane + (size_t)y * n + j] = acc[k];
  }
}

__global__ void k_xys_add(const double* __restrict__ part, double* __restrict__ xys, SgsGrid G, int nacc) {
  const size_t plane = (size_t)G.nyp * G.nx;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= plane) return;
  for (int k = 0; k < nacc; ++k) {
    double s = 0.0;
    for (int grp = 0; grp < XYS_GROUPS; ++grp) s += part[((size_t)grp * XYS_NACC_P + k) * plane + i];
    xys[(size_t)(xys_entry(k) - 1) * plane + i] += s;
  }
}

__global__ void k_xys_minmax(const double* __restrict__ uphys, double* __restrict__ xys, SgsGrid G) {
  const size_t plane = (size_t)G.nyp * G.nx;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= plane) return;
  const int y = (int)(i / G.nx), x = (int)(i - (size_t)y * G.nx);
  const double* u = uphys + (size_t)y * G.nz * G.nx + x;
  double ut = 0.0;
  for (int m = 0; m < G.nz; ++m) ut = ut + u[(size_t)m * G.nx];
  ut = ut / (double)G.nz;
  double umin = xys[(size_t)42 * plane + i], umax = xys[(size_t)43 * plane + i];
  for (int m = 0; m < G.nz; ++m) {
    const double d = u[(size_t)m * G.nx] - ut;
    umax = fmax(umax, d);
    umin = fmin(umin, d);
  }
  xys[(size_t)42 * plane + i] = umin;
  xys[(size_t)43 * plane + i] = umax;
}

// Training sample of the learned SGS model from the resolved state (the box
// filtering of the high-resolution channel that produces its data): on the
// nx x nz grid, per y-plane, the top-hat average over cells of f x f points
// (x in [f X, f X + f), z in [f Z, f Z + f)) of u_i, of the nine gradients
// du_i/dx_j and of the products u_i u_j.  Per coarse point, features[10] =
// the nine filtered gradients (i-major) and the wall distance 1 - |y|, and
// targets[6] = tau_ij = <u_i u_j> - <u_i> <u_j> (11 12 13 22 23 33): the
// inputs and the output of the model of sgs_mlp.cuh, unscaled.  One CTA per
// (Z, y), blockDim >= nx / f; reads the spectral fields of k_xys_zinv.
__global__ void __launch_bounds__(512) k_box_sample(const double2* __restrict__ spec, SgsGrid G, FFTPlan plan,
                                                    const double2* __restrict__ tw, int f,
                                                    float* __restrict__ features, float* __restrict__ targets) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* bA = reinterpret_cast<double2*>(smem_raw);
  double2* bB = bA + (size_t)G.nx * XYS_NC;
  const int Z = blockIdx.x, y = blockIdx.y;
  const int n = G.nx, nxc = G.nx / f, nzc = G.nz / f;
  const int X = threadIdx.x;
  const size_t fs = (size_t)G.nyp * G.nz * G.nx2;
  double acc[18];
#pragma unroll
  for (int k = 0; k < 18; ++k) acc[k] = 0.0;
  for (int rr = 0; rr < f; ++rr) {
    const size_t row = ((size_t)y * G.nz + (size_t)f * Z + rr) * G.nx2;
    for (int t = threadIdx.x; t < n * XYS_NC; t += blockDim.x) {
      const int k = t / XYS_NC, cc = t - XYS_NC * (t / XYS_NC);
      const double2* a = spec + (size_t)(2 * cc) * fs + row;
      const double2* b = (2 * cc + 1 < XYS_NF) ? spec + (size_t)(2 * cc + 1) * fs + row : nullptr;
      bA[k * XYS_NC + cc] = sgs_pair(a, b, k, n, G.nx2);
    }
    __syncthreads();
    const double2* res = fft_columns<double, XYS_NC>(bA, bB, plan, tw, +1);
    if (X < nxc) {
      for (int xx = 0; xx < f; ++xx) {
        const int j = f * X + xx;
        double q[16];
#pragma unroll
        for (int cc = 0; cc < XYS_NC; ++cc) {
          const double2 zv = res[j * XYS_NC + cc];
          q[2 * cc] = zv.x;
          q[2 * cc + 1] = zv.y;
        }
        const double u = q[0], v = q[1], w = q[2];
        acc[0] += u;
        acc[1] += v;
        acc[2] += w;
#pragma unroll
        for (int k = 0; k < 9; ++k) acc[3 + k] += q[6 + k];
        acc[12] += u * u;
        acc[13] += u * v;
        acc[14] += u * w;
        acc[15] += v * v;
        acc[16] += v * w;
        acc[17] += w * w;
      }
    }
    __syncthreads();
  }
  if (X < nxc) {
    const double inv = 1.0 / ((double)f * (double)f);
    const double ub[3] = {acc[0] * inv, acc[1] * inv, acc[2] * inv};
    const size_t pt = ((size_t)y * nzc + Z) * nxc + X;
    float* fo = features + pt * 10;
#pragma unroll
    for (int k = 0; k < 9; ++k) fo[k] = (float)(acc[3 + k] * inv);
    const double eta = cos(3.14159265358979323846 * (double)y / (double)(G.nyp - 1));
    fo[9] = (float)(1.0 - fabs(eta));
    float* to = targets + pt * 6;
    const int pi_[6] = {0, 0, 0, 1, 1, 2}, pj_[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int c = 0; c < 6; ++c) to[c] = (float)(acc[12 + c] * inv - ub[pi_[c]] * ub[pj_[c]]);
  }
}

}  // namespace sb
