// Eddy-viscosity large-eddy model on the device (iles = 2; iles = 3 feeds it
// the high-pass filtered fields, see k_sgs_zinv and k_sgs_xpass1): the Smagorinsky
// stress tau_ij = -2 C Delta^2 |S| S_ij with the dynamic (Germano/Lilly)
// coefficient C, its divergence sigma_i = d tau_ij / dx_j, and -sigma added
// to H in step 2.  The reference computes tau plane by plane in bla/les.f
// (before nonlinbl, every substep), sigma pencil by pencil in
// bla/sgs_stress.f, and adds it in bla/nonlinbl.f:1011-1048.
//
// Grid: the stored modes on the nx x nz grid (no 3/2 padding), as les.f's
// getxz(...,0,...) and its length-nx / length-nz transforms.
//
//   k_sgs_zinv   per plane and kx block: u, v, w and the six strain-rate
//                components S_ij (from u, v, w, omega_x, omega_z: x and z
//                derivatives spectrally, y derivatives from the vorticity and
//                continuity, les.f:288-327), oddball zeroed, inverse z FFT
//   k_sgs_xpass1 per plane and z row: inverse x FFT (two real fields per
//                complex FFT), |S|; the 21 fields the test filter acts on
//                (M_ij parts, L_ij parts, S_ij, u_i; les.f:709-771), forward
//                x FFT, keep kx < nx/4 (filter_cutoff.f)
//   k_sgs_zfilt  forward z FFT, keep |kz| <= nz/4, inverse z FFT
//   k_sgs_xpass2 inverse x FFT of the filtered fields, L_ij and M_ij
//                (les.f:783-881), per-point M:L and M:M
//   k_sgs_coef   C(x, y) = max(<M:L>_z / (2 <M:M>_z), 0), the average over z
//                (les.f:1385-1480, ineg = 1 clipping, zero at the walls)
//   k_sgs_tau_x  tau_ij / (nx nz) (les.f:1489-1560), forward x FFT
//   k_sgs_zfwd   forward z FFT, oddball zeroed: tau in the state layout
//   k_sgs_backscatter (learned model) per plane: the plane sums of
//                tau_ij S_ij and |tau_ij S_ij| of the network's stress, and
//                the plane's switch to the eddy-viscosity model
//   k_sgs_sigma  per pencil, on Chebyshev coefficients of tau:
//                sigma_i = i alpha tau_i1 + i beta tau_i3 + D tau_i2
//                (bla/sgs_stress.f)
//
// All arithmetic is FP64 whatever the state storage.
#pragma once
#include "fft.cuh"
#include "layout.cuh"
#include "step3.cuh"

namespace sb {

struct SgsBufs {
  double2* spec9;   // [9][nyp][nz][nx/2]   z physical, x spectral
  double* phys10;   // [10][nyp][nz][nx]    u v w S11 S12 S13 S22 S23 S33 |S|
  double2* filt21;  // [21][nyp][nz][nx/4]  test-filtered fields, x spectral
  double* numden;   // [2][nyp][nz][nx]     M:L and M:M per point
  double* cxy;      // [nyp][nx]            C(x, y)
  double2* tauz6;   // [6][nyp][nz][nx/2]   tau, z physical, x spectral
  double2* tau;     // [6][nyp][NP]         tau, state layout
  // learned model with the per-plane fallback: planes y with plane_on[y] != 0
  // take the eddy-viscosity stress, the others the network's; the
  // eddy-viscosity kernels skip the other planes.  nullptr: every plane
  // (the plain eddy-viscosity model).
  const int* plane_on;
};

__device__ __forceinline__ bool sgs_plane_off(const SgsBufs& B, int y) {
  return B.plane_on != nullptr && B.plane_on[y] == 0;
}

struct SgsGrid {
  int nx, nz, nx2, nx4, nyp, NP, zodd;
};

// Field set 0: u, v, w, S11, S12, S13, S22, S23, S33; field set 1: the nine
// gradients du_i/dx_j (i-major), spectral at (y, iz, kx)
template <class V>
__device__ __forceinline__ double2 sgs_spec_field(const V* st, size_t slot, size_t off, int f, double a, double b,
                                                  int set) {
  auto ld = [&](int s) { const V q = st[(size_t)s * slot + off]; return double2{(double)q.x, (double)q.y}; };
  // i k q = (-k q.y, k q.x)
  if (set == 1) {
    switch (f) {
      case 0: { const double2 u = ld(0); return double2{-a * u.y, a * u.x}; }
      case 1: {
        const double2 v = ld(1), oz = ld(4);
        return double2{-a * v.y - oz.x, a * v.x - oz.y};
      }
      case 2: { const double2 u = ld(0); return double2{-b * u.y, b * u.x}; }
      case 3: { const double2 v = ld(1); return double2{-a * v.y, a * v.x}; }
      case 4: {
        const double2 u = ld(0), w = ld(2);
        return double2{a * u.y + b * w.y, -a * u.x - b * w.x};
      }
      case 5: { const double2 v = ld(1); return double2{-b * v.y, b * v.x}; }
      case 6: { const double2 w = ld(2); return double2{-a * w.y, a * w.x}; }
      case 7: {
        const double2 v = ld(1), ox = ld(3);
        return double2{ox.x - b * v.y, ox.y + b * v.x};
      }
      default: { const double2 w = ld(2); return double2{-b * w.y, b * w.x}; }
    }
  }
  switch (f) {
    case 0: return ld(0);
    case 1: return ld(1);
    case 2: return ld(2);
    case 3: { const double2 u = ld(0); return double2{-a * u.y, a * u.x}; }
    case 4: {
      // S12 = (dv/dx + du/dy)/2, du/dy = dv/dx - omega_z
      const double2 v = ld(1), oz = ld(4);
      const double2 dvdx{-a * v.y, a * v.x};
      return double2{.5 * (dvdx.x + (dvdx.x - oz.x)), .5 * (dvdx.y + (dvdx.y - oz.y))};
    }
    case 5: {
      const double2 u = ld(0), w = ld(2);
      return double2{.5 * (-a * w.y + -b * u.y), .5 * (a * w.x + b * u.x)};
    }
    case 6: {
      // dv/dy = -du/dx - dw/dz
      const double2 u = ld(0), w = ld(2);
      return double2{a * u.y + b * w.y, -a * u.x - b * w.x};
    }
    case 7: {
      // S23 = (dv/dz + dw/dy)/2, dw/dy = omega_x + dv/dz
      const double2 v = ld(1), ox = ld(3);
      const double2 dvdz{-b * v.y, b * v.x};
      return double2{.5 * (dvdz.x + (ox.x + dvdz.x)), .5 * (dvdz.y + (ox.y + dvdz.y))};
    }
    default: { const double2 w = ld(2); return double2{-b * w.y, b * w.x}; }
  }
}

// sf != nullptr (field set 0): the strain-rate fields 3..8 from the fields
// of sf (the dynamic HPF model: u from the state, S_ij of the high-pass
// filtered field), u, v, w from st.
template <class V, int KB>
__global__ void k_sgs_zinv(const V* __restrict__ st, SgsBufs B, SgsGrid G, FFTPlan plan,
                           const double2* __restrict__ tw, const double* __restrict__ alfa,
                           const double* __restrict__ beta, int set, const double2* __restrict__ sf) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* b0 = reinterpret_cast<double2*>(smem_raw);
  double2* b1 = b0 + (size_t)G.nz * KB;
  const int y = blockIdx.y;
  if (set == 0 && sgs_plane_off(B, y)) return;
  const int kx0 = blockIdx.x * KB;
  const size_t slot = (size_t)G.nyp * G.NP;
  for (int f = 0; f < 9; ++f) {
    for (int t = threadIdx.x; t < G.nz * KB; t += blockDim.x) {
      const int iz = t / KB;
      const int kx = kx0 + t - iz * KB;
      double2 val{0.0, 0.0};
      if (kx < G.nx2 && iz != G.zodd) {
        const size_t off = (size_t)y * G.NP + (size_t)iz * G.nx2 + kx;
        val = (sf != nullptr && f >= 3) ? sgs_spec_field(sf, slot, off, f, alfa[kx], beta[iz], set)
                                        : sgs_spec_field(st, slot, off, f, alfa[kx], beta[iz], set);
      }
      b0[t] = val;
    }
    __syncthreads();
    double2* res = fft_columns<double, KB>(b0, b1, plan, tw, +1);
    for (int t = threadIdx.x; t < G.nz * KB; t += blockDim.x) {
      const int m = t / KB;
      const int kx = kx0 + t - m * KB;
      if (kx < G.nx2) B.spec9[(((size_t)f * G.nyp + y) * G.nz + m) * G.nx2 + kx] = res[t];
    }
    __syncthreads();
  }
}

// Hermitian completion of the half spectra a, b (kx < nk, the rest zero) of
// two real rows into the spectrum of a + i b at index k of a length-n FFT.
__device__ __forceinline__ double2 sgs_pair(const double2* a, const double2* b, int k, int n, int nk) {
  if (k == 0) return double2{a ? a[0].x : 0.0, b ? b[0].x : 0.0};
  if (k < nk) {
    const double2 p = a ? a[k] : double2{0.0, 0.0}, q = b ? b[k] : double2{0.0, 0.0};
    return double2{p.x - q.y, p.y + q.x};
  }
  if (k > n - nk) {
    const int kk = n - k;
    const double2 p = a ? a[kk] : double2{0.0, 0.0}, q = b ? b[kk] : double2{0.0, 0.0};
    return double2{p.x + q.y, q.x - p.y};
  }
  return double2{0.0, 0.0};
}

// sqrt(2 (S11^2 + S22^2 + S33^2) + 4 (S12^2 + S13^2 + S23^2)), les.f:660-665
__device__ __forceinline__ double sgs_sabs(const double* s) {
  return sqrt(2. * (s[0] * s[0] + s[3] * s[3] + s[5] * s[5]) + 4. * (s[1] * s[1] + s[2] * s[2] + s[4] * s[4]));
}

// One z row per CTA.  Shared memory: two buffers of 11 columns x nx.
// s2 != nullptr: the test filter's B_ij parts are these six physical fields
// (the dynamic HPF model: the strain of the secondary high-pass filtered
// field, bla/les.f:1031-1250) instead of S_ij.
__global__ void k_sgs_xpass1(SgsBufs B, SgsGrid G, FFTPlan plan, const double2* __restrict__ tw,
                             const double* __restrict__ delta2, const double* __restrict__ s2) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NC = 11;
  double2* bA = reinterpret_cast<double2*>(smem_raw);
  double2* bB = bA + (size_t)G.nx * NC;
  const int m = blockIdx.x, y = blockIdx.y;
  if (sgs_plane_off(B, y)) return;
  const int n = G.nx;
  const size_t fs9 = (size_t)G.nyp * G.nz * G.nx2;
  const size_t row = ((size_t)y * G.nz + m) * G.nx2;
  // five complex FFTs carry the nine real rows (u+iv, w+iS11, S12+iS13, S22+iS23, S33)
  for (int t = threadIdx.x; t < n * 5; t += blockDim.x) {
    const int k = t / 5, c = t - 5 * (t / 5);
    const double2* a = B.spec9 + (size_t)(2 * c) * fs9 + row;
    const double2* b = (2 * c + 1 < 9) ? B.spec9 + (size_t)(2 * c + 1) * fs9 + row : nullptr;
    bA[k * 5 + c] = sgs_pair(a, b, k, n, G.nx2);
  }
  __syncthreads();
  double2* res = fft_columns<double, 5>(bA, bB, plan, tw, +1);
  double2* oth = (res == bA) ? bB : bA;
  const double d2 = delta2[y];
  const size_t fs10 = (size_t)G.nyp * G.nz * G.nx;
  const size_t prow = ((size_t)y * G.nz + m) * G.nx;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double q[9];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const double2 z = res[j * 5 + c];
      q[2 * c] = z.x;
      if (2 * c + 1 < 9) q[2 * c + 1] = z.y;
    }
    const double u = q[0], v = q[1], w = q[2];
    const double* s = q + 3;  // S11 S12 S13 S22 S23 S33
    const double sabs = sgs_sabs(s);
#pragma unroll
    for (int f = 0; f < 9; ++f) B.phys10[(size_t)f * fs10 + prow + j] = q[f];
    B.phys10[(size_t)9 * fs10 + prow + j] = sabs;
    const double dr = sabs * d2;
    double r[22];
    for (int l = 0; l < 6; ++l) r[l] = -s[l] * dr;  // M parts
    r[6] = -u * u;                                   // L parts
    r[7] = -v * u;
    r[8] = -w * u;
    r[9] = -v * v;
    r[10] = -w * v;
    r[11] = -w * w;
    for (int l = 0; l < 6; ++l) r[12 + l] = s2 ? s2[(size_t)l * fs10 + prow + j] : s[l];  // B = S (or S of H2 u)
    r[18] = u;
    r[19] = v;
    r[20] = w;
    r[21] = 0.0;
#pragma unroll
    for (int c = 0; c < NC; ++c) oth[j * NC + c] = double2{r[2 * c], r[2 * c + 1]};
  }
  __syncthreads();
  double2* fres = fft_columns<double, NC>(oth, res, plan, tw, -1);
  const size_t fs21 = (size_t)G.nyp * G.nz * G.nx4;
  const size_t frow = ((size_t)y * G.nz + m) * G.nx4;
  for (int t = threadIdx.x; t < G.nx4 * NC; t += blockDim.x) {
    const int k = t / NC, c = t - NC * (t / NC);
    const double2 a = fres[k * NC + c];
    const double2 b = fres[((n - k) % n) * NC + c];
    // spectra of the real and imaginary rows
    B.filt21[(size_t)(2 * c) * fs21 + frow + k] = double2{(a.x + b.x) * .5, (a.y - b.y) * .5};
    if (2 * c + 1 < 21) B.filt21[(size_t)(2 * c + 1) * fs21 + frow + k] = double2{(a.y + b.y) * .5, (b.x - a.x) * .5};
  }
}

// The nine spec9 rows of one z row back to physical x: fields f0..8 into
// out[f - f0] (the learned model's gradients: out = phys10, f0 = 0; the
// dynamic HPF model's secondary strain: f0 = 3).
__global__ void k_sgs_xinv9(SgsBufs B, SgsGrid G, FFTPlan plan, const double2* __restrict__ tw,
                            double* __restrict__ out, int f0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* bA = reinterpret_cast<double2*>(smem_raw);
  double2* bB = bA + (size_t)G.nx * 5;
  const int m = blockIdx.x, y = blockIdx.y;
  const int n = G.nx;
  const size_t fs9 = (size_t)G.nyp * G.nz * G.nx2;
  const size_t row = ((size_t)y * G.nz + m) * G.nx2;
  for (int t = threadIdx.x; t < n * 5; t += blockDim.x) {
    const int k = t / 5, c = t - 5 * (t / 5);
    const double2* a = B.spec9 + (size_t)(2 * c) * fs9 + row;
    const double2* b = (2 * c + 1 < 9) ? B.spec9 + (size_t)(2 * c + 1) * fs9 + row : nullptr;
    bA[k * 5 + c] = sgs_pair(a, b, k, n, G.nx2);
  }
  __syncthreads();
  double2* res = fft_columns<double, 5>(bA, bB, plan, tw, +1);
  const size_t fs10 = (size_t)G.nyp * G.nz * G.nx;
  const size_t prow = ((size_t)y * G.nz + m) * G.nx;
  for (int t = threadIdx.x; t < n * 5; t += blockDim.x) {
    const int j = t / 5, c = t - 5 * (t / 5);
    const double2 z = res[j * 5 + c];
    if (2 * c >= f0) out[(size_t)(2 * c - f0) * fs10 + prow + j] = z.x;
    if (2 * c + 1 < 9 && 2 * c + 1 >= f0) out[(size_t)(2 * c + 1 - f0) * fs10 + prow + j] = z.y;
  }
}

// Test filter in z on the kept kx < nx/4 columns: forward FFT, zero
// nz/4 < |kz| (filter_cutoff.f: z = nz/4+2 .. nz-nz/4 zeroed), inverse FFT.
template <int KB>
__global__ void k_sgs_zfilt(SgsBufs B, SgsGrid G, FFTPlan plan, const double2* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* b0 = reinterpret_cast<double2*>(smem_raw);
  double2* b1 = b0 + (size_t)G.nz * KB;
  const int y = blockIdx.y;
  if (sgs_plane_off(B, y)) return;
  const int kx0 = blockIdx.x * KB;
  const size_t fs21 = (size_t)G.nyp * G.nz * G.nx4;
  const int zlo = G.nz / 4 + 1, zhi = G.nz - G.nz / 4 - 1;
  for (int f = 0; f < 21; ++f) {
    double2* fld = B.filt21 + (size_t)f * fs21 + (size_t)y * G.nz * G.nx4;
    for (int t = threadIdx.x; t < G.nz * KB; t += blockDim.x) {
      const int m = t / KB;
      const int kx = kx0 + t - m * KB;
      b0[t] = (kx < G.nx4) ? fld[(size_t)m * G.nx4 + kx] : double2{0.0, 0.0};
    }
    __syncthreads();
    double2* res = fft_columns<double, KB>(b0, b1, plan, tw, -1);
    for (int t = threadIdx.x; t < G.nz * KB; t += blockDim.x) {
      const int m = t / KB;
      if (m >= zlo && m <= zhi) res[t] = double2{0.0, 0.0};
    }
    __syncthreads();
    double2* oth = (res == b0) ? b1 : b0;
    double2* back = fft_columns<double, KB>(res, oth, plan, tw, +1);
    for (int t = threadIdx.x; t < G.nz * KB; t += blockDim.x) {
      const int m = t / KB;
      const int kx = kx0 + t - m * KB;
      if (kx < G.nx4) fld[(size_t)m * G.nx4 + kx] = back[t];
    }
    __syncthreads();
  }
}

// Inverse x FFT of the 21 test-filtered fields (divided by nx nz as
// filter_cutoff.f does), then L_ij, M_ij and the per-point contractions.
__global__ void k_sgs_xpass2(SgsBufs B, SgsGrid G, FFTPlan plan, const double2* __restrict__ tw,
                             const double* __restrict__ delta2) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NC = 11;
  double2* bA = reinterpret_cast<double2*>(smem_raw);
  double2* bB = bA + (size_t)G.nx * NC;
  const int m = blockIdx.x, y = blockIdx.y;
  if (sgs_plane_off(B, y)) return;
  const int n = G.nx;
  const size_t fs21 = (size_t)G.nyp * G.nz * G.nx4;
  const size_t frow = ((size_t)y * G.nz + m) * G.nx4;
  for (int t = threadIdx.x; t < n * NC; t += blockDim.x) {
    const int k = t / NC, c = t - NC * (t / NC);
    const double2* a = B.filt21 + (size_t)(2 * c) * fs21 + frow;
    const double2* b = (2 * c + 1 < 21) ? B.filt21 + (size_t)(2 * c + 1) * fs21 + frow : nullptr;
    bA[k * NC + c] = sgs_pair(a, b, k, n, G.nx4);
  }
  __syncthreads();
  double2* res = fft_columns<double, NC>(bA, bB, plan, tw, +1);
  const double inv = 1.0 / (double)(G.nx * G.nz);
  const double gd2 = pow(4., 2. / 3.) * delta2[y];
  const size_t fs10 = (size_t)G.nyp * G.nz * G.nx;
  const size_t prow = ((size_t)y * G.nz + m) * G.nx;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double r[22];
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const double2 z = res[j * NC + c];
      r[2 * c] = z.x * inv;
      r[2 * c + 1] = z.y * inv;
    }
    const double* mt = r;       // filtered M parts
    const double* lt = r + 6;   // filtered -u_i u_j
    const double* bt = r + 12;  // filtered S
    const double u = r[18], v = r[19], w = r[20];
    double L[6], M[6];
    L[0] = lt[0] + u * u;
    L[1] = lt[1] + v * u;
    L[2] = lt[2] + w * u;
    L[3] = lt[3] + v * v;
    L[4] = lt[4] + w * v;
    L[5] = lt[5] + w * w;
    const double dr = gd2 * sgs_sabs(bt);
    for (int l = 0; l < 6; ++l) M[l] = mt[l] + bt[l] * dr;
    const double num = M[0] * L[0] + M[3] * L[3] + M[5] * L[5] + 2. * (M[1] * L[1] + M[2] * L[2] + M[4] * L[4]);
    const double den = M[0] * M[0] + M[3] * M[3] + M[5] * M[5] + 2. * (M[1] * M[1] + M[2] * M[2] + M[4] * M[4]);
    B.numden[prow + j] = num;
    B.numden[fs10 + prow + j] = den;
  }
}

// C(x, y) from the z averages (les.f:1385-1480).  cs > 0: fixed C = cs^2.
// ineg: 0 no clipping, 1 C >= 0 and zero at the walls, 2 zero at the walls
// (the nu_t + nu >= 0 clip follows in k_sgs_tau_x).
__global__ void k_sgs_coef(SgsBufs B, SgsGrid G, double cs, int ineg) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= G.nx || sgs_plane_off(B, y)) return;
  double c;
  if (cs != 0.0) {
    c = cs * cs;
  } else {
    const size_t plane = (size_t)G.nyp * G.nz * G.nx;
    double num = 0.0, den = 0.0;
    for (int m = 0; m < G.nz; ++m) {
      const size_t o = ((size_t)y * G.nz + m) * G.nx + x;
      num += B.numden[o];
      den += B.numden[plane + o];
    }
    const bool wall = (y == 0 || y == G.nyp - 1);
    if (ineg == 1)
      c = wall ? 0.0 : fmax(.5 * num / den, 0.);
    else if (ineg == 2)
      c = wall ? 0.0 : .5 * num / den;
    else
      c = .5 * num / den;
  }
  B.cxy[(size_t)y * G.nx + x] = c;
}

// tau_ij / (nx nz) = -2 C Delta^2 |S| S_ij / (nx nz) in physical space, then
// the forward x FFT (three complex FFTs for the six real rows).
// tau_phys != nullptr: the stress is given in physical space ([6][nyp*nz*nx],
// the learned model) instead of -2 C Delta^2 |S| S_ij, except on the planes
// that B.plane_on switches to the eddy-viscosity model.
__global__ void k_sgs_tau_x(SgsBufs B, SgsGrid G, FFTPlan plan, const double2* __restrict__ tw,
                            const double* __restrict__ delta2, double re, int ineg,
                            const double* __restrict__ tau_phys) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* bA = reinterpret_cast<double2*>(smem_raw);
  double2* bB = bA + (size_t)G.nx * 3;
  const int m = blockIdx.x, y = blockIdx.y;
  const int n = G.nx;
  const size_t fs10 = (size_t)G.nyp * G.nz * G.nx;
  const size_t prow = ((size_t)y * G.nz + m) * G.nx;
  const double gd2 = 1. / (double)(G.nx * G.nz);
  const double d2 = delta2[y];
  const bool learned = tau_phys != nullptr && (B.plane_on == nullptr || B.plane_on[y] == 0);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double t[6];
    if (learned) {
      for (int l = 0; l < 6; ++l) t[l] = tau_phys[(size_t)l * fs10 + prow + j] * gd2;
    } else {
      double dr = B.cxy[(size_t)y * G.nx + j] * B.phys10[9 * fs10 + prow + j] * d2;
      if (ineg == 2 && dr < -1. / re) dr = -1. / re;
      const double d1 = -2. * dr * gd2;
      for (int l = 0; l < 6; ++l) t[l] = d1 * B.phys10[(size_t)(3 + l) * fs10 + prow + j];
    }
    for (int c = 0; c < 3; ++c) bA[j * 3 + c] = double2{t[2 * c], t[2 * c + 1]};
  }
  __syncthreads();
  double2* res = fft_columns<double, 3>(bA, bB, plan, tw, -1);
  const size_t fs = (size_t)G.nyp * G.nz * G.nx2;
  const size_t row = ((size_t)y * G.nz + m) * G.nx2;
  for (int t = threadIdx.x; t < G.nx2 * 3; t += blockDim.x) {
    const int k = t / 3, c = t - 3 * (t / 3);
    const double2 a = res[k * 3 + c];
    const double2 b = res[((n - k) % n) * 3 + c];
    B.tauz6[(size_t)(2 * c) * fs + row + k] = double2{(a.x + b.x) * .5, (a.y - b.y) * .5};
    B.tauz6[(size_t)(2 * c + 1) * fs + row + k] = double2{(a.y + b.y) * .5, (b.x - a.x) * .5};
  }
}

// Per-plane switch of the learned model (no counterpart in the reference):
// one CTA per plane y sums, in a fixed order, P = tau_ij S_ij and
// |tau_ij S_ij| over the plane's nz x nx points (tau the network's physical
// stress, S_ij = (du_i/dx_j + du_j/dx_i) / 2 from the nine gradients in
// phys10 fields 0-8).  P > 0 is backscatter (energy from the SGS to the
// resolved scales, the SGS dissipation -tau_ij S_ij being negative).  The
// plane switches to the eddy-viscosity model when sum P > bound * sum |P|
// (bound in [-1, 1]: 1 never, below -1 always).  sums[2 y], sums[2 y + 1]
// keep the two sums for diagnostics.
__global__ void __launch_bounds__(1024) k_sgs_backscatter(SgsBufs B, SgsGrid G, const double* __restrict__ tau,
                                                         double bound, int* __restrict__ plane_on,
                                                         double* __restrict__ sums) {
  const int y = blockIdx.x;
  const size_t plane = (size_t)G.nz * G.nx;
  const size_t fs = (size_t)G.nyp * plane;
  const size_t o0 = (size_t)y * plane;
  double p = 0.0, pa = 0.0;
  for (size_t i = threadIdx.x; i < plane; i += blockDim.x) {
    const size_t o = o0 + i;
    double g[9], t[6];
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = B.phys10[(size_t)k * fs + o];
#pragma unroll
    for (int k = 0; k < 6; ++k) t[k] = tau[(size_t)k * fs + o];
    const double s11 = g[0], s22 = g[4], s33 = g[8];
    const double s12 = .5 * (g[1] + g[3]), s13 = .5 * (g[2] + g[6]), s23 = .5 * (g[5] + g[7]);
    const double q = t[0] * s11 + t[3] * s22 + t[5] * s33 + 2. * (t[1] * s12 + t[2] * s13 + t[4] * s23);
    p += q;
    pa += fabs(q);
  }
  // fixed-order reduction: warps by shuffles, then warp 0 over the warps
  __shared__ double rp[32], ra[32];
  for (int d = 16; d > 0; d >>= 1) {
    p += __shfl_down_sync(0xffffffffu, p, d);
    pa += __shfl_down_sync(0xffffffffu, pa, d);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    rp[warp] = p;
    ra[warp] = pa;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sp = 0.0, sa = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      sp += rp[w];
      sa += ra[w];
    }
    plane_on[y] = (sp > bound * sa) ? 1 : 0;
    sums[2 * y] = sp;
    sums[2 * y + 1] = sa;
  }
}

// Forward z FFT of tau; the oddball kz = -nz/2 is zeroed (les.f:1576-1590).
template <int KB>
__global__ void k_sgs_zfwd(SgsBufs B, SgsGrid G, FFTPlan plan, const double2* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* b0 = reinterpret_cast<double2*>(smem_raw);
  double2* b1 = b0 + (size_t)G.nz * KB;
  const int y = blockIdx.y;
  const int kx0 = blockIdx.x * KB;
  const size_t fs = (size_t)G.nyp * G.nz * G.nx2;
  const size_t slot = (size_t)G.nyp * G.NP;
  for (int f = 0; f < 6; ++f) {
    for (int t = threadIdx.x; t < G.nz * KB; t += blockDim.x) {
      const int m = t / KB;
      const int kx = kx0 + t - m * KB;
      b0[t] = (kx < G.nx2) ? B.tauz6[(size_t)f * fs + ((size_t)y * G.nz + m) * G.nx2 + kx] : double2{0.0, 0.0};
    }
    __syncthreads();
    double2* res = fft_columns<double, KB>(b0, b1, plan, tw, -1);
    for (int t = threadIdx.x; t < G.nz * KB; t += blockDim.x) {
      const int iz = t / KB;
      const int kx = kx0 + t - iz * KB;
      if (kx < G.nx2)
        B.tau[(size_t)f * slot + (size_t)y * G.NP + (size_t)iz * G.nx2 + kx] =
            (iz == G.zodd) ? double2{0.0, 0.0} : res[t];
    }
    __syncthreads();
  }
}

// sigma_i on Chebyshev coefficients (bla/sgs_stress.f): tc = Chebyshev
// coefficients of tau [6][nyp][NP], sc = output [3][nyp][NP].  One warp per
// pencil: the x and z derivatives row by row, and D tau_i2 -- the Chebyshev
// derivative b_j = sum over k > j with k - j odd of 2 k a_k, b_0 halved (the
// closed form of the bla/dcheb.f recurrence) -- as suffix sums: each lane
// sums its block of rows by parity, the warp scans the block sums, and each
// lane walks its rows down from its carry.
__global__ void __launch_bounds__(128) k_sgs_sigma(const double2* __restrict__ tc, double2* __restrict__ sc,
                                                   SgsGrid G, const double* __restrict__ alfa,
                                                   const double* __restrict__ beta) {
  const int lane = threadIdx.x & 31;
  const int p = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  if (p >= G.NP) return;  // the whole warp leaves together
  const int kx = p % G.nx2, iz = p / G.nx2;
  const double a = alfa[kx], b = beta[iz];
  const size_t fld = (size_t)G.nyp * G.NP;
  const int n = G.nyp;
  const int per = (n + 31) / 32;
  const int j0 = min(n, lane * per), j1 = min(n, j0 + per);
  // sigma_1 = i a tau11 + i b tau13 + D tau12; sigma_2 = i a tau12 + i b tau23
  // + D tau22; sigma_3 = i a tau13 + i b tau33 + D tau23
  // tau slots: i a tau_(i,1), i b tau_(i,3), D tau_(i,2) of row i (selects,
  // so no index table goes to local memory)
  for (int i = 0; i < 3; ++i) {
    const int cx = i, cy = (i == 0) ? 1 : (i == 1 ? 3 : 4), cz = (i == 0) ? 2 : (i == 1 ? 4 : 5);
    const double2* ty = tc + (size_t)cy * fld + p;
    // this lane's block sums of 2 k a_k, k even / k odd
    double2 se{0.0, 0.0}, so{0.0, 0.0};
    for (int k = j0; k < j1; ++k) {
      const double2 v = ty[(size_t)k * G.NP];
      const double f = 2.0 * (double)k;
      if (k & 1) {
        so.x += f * v.x;
        so.y += f * v.y;
      } else {
        se.x += f * v.x;
        se.y += f * v.y;
      }
    }
    // carry = sums over the rows of the lanes above this one
    double2 ce = se, co = so;  // inclusive suffix sums after the scan
    for (int d = 1; d < 32; d <<= 1) {
      const double ex = __shfl_down_sync(0xffffffffu, ce.x, d), ey = __shfl_down_sync(0xffffffffu, ce.y, d);
      const double ox = __shfl_down_sync(0xffffffffu, co.x, d), oy = __shfl_down_sync(0xffffffffu, co.y, d);
      if (lane + d < 32) {
        ce.x += ex;
        ce.y += ey;
        co.x += ox;
        co.y += oy;
      }
    }
    double2 Se{ce.x - se.x, ce.y - se.y}, So{co.x - so.x, co.y - so.y};  // sums over k >= j1
    for (int j = j1 - 1; j >= j0; --j) {
      const size_t o = (size_t)j * G.NP + p;
      const double2 v = ty[(size_t)j * G.NP];
      double2 d = (j & 1) ? Se : So;  // k > j of the other parity
      if (j == 0) d = double2{0.5 * d.x, 0.5 * d.y};
      const double2 tx = tc[(size_t)cx * fld + o];
      const double2 tz = tc[(size_t)cz * fld + o];
      sc[(size_t)i * fld + o] = double2{-a * tx.y - b * tz.y + d.x, a * tx.x + b * tz.x + d.y};
      const double f = 2.0 * (double)j;
      if (j & 1) {
        So.x += f * v.x;
        So.y += f * v.y;
      } else {
        Se.x += f * v.x;
        Se.y += f * v.y;
      }
    }
  }
}

}  // namespace sb
