// Step 2 of the RK substep: the nonlinear term H = u x omega in physical space
// (the work bla/nonlinbl.f does plane by plane).
//
//   k_zinv : per xz-plane and block of kx columns: read u, v, w, omega_x,
//            omega_z (and form omega_y = i beta u - i alpha w) from the
//            spectral state, zero-pad kz 2/3 -> 3/2 grid (pad folded into the
//            load: the zero band and the oddball mode are never read), inverse
//            complex FFT over z.
//   k_xpass: per xz-plane and block of z rows: Hermitian-complete two fields
//            per complex FFT (u+iv, w+i omega_x, omega_y+i omega_z), inverse
//            FFT over x, form H and the CFL number in registers, forward FFT
//            of (H1+iH2) and H3, split the spectra and keep kx < nx/2.
//   k_zfwd : forward complex FFT over z, keep the nz stored kz modes
//            (truncation folded into the store) and write H into state slots
//            1-3, exactly where the reference's putxz puts it.
//
// Normalisation follows the reference: synthesis and analysis are both
// unnormalised, so H carries the factor nxp*nzp that the Chebyshev transform
// of step 3 removes.
#pragma once
#include "fft.cuh"
#include "layout.cuh"

namespace sb {

// The z transforms work through their fields one after another, and a
// field's first loads can only start after the previous field's barrier:
// while a field is transformed, its successor's rows of the CTA's columns are
// prefetched into L2 (no registers held, no effect on the values).  FP64
// transforms only: at 384x193x384 the FP64 z-inverse went 1.117 -> 1.024 ms
// and the z-forward 0.624 -> 0.553, the FP32 z-inverse 0.507 -> 0.546.
#ifndef SB_Z_PREFETCH
#define SB_Z_PREFETCH 1
#endif
__device__ __forceinline__ void z_prefetch_l2(const void* ptr) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(ptr)));
}

// drop_mean: leave out the kx = kz = 0 mode (the mean profiles U, W,
// Omega_x, Omega_z), which the mixed-precision path adds back analytically.
// N > 0: the z length g.nzp is N, transformed with the compile-time plan by
// NT threads per CTA; N = 0: runtime plan, any block size.
// (the FP64 fixed-length variant is held to three CTAs per SM: unbounded it
// takes ~130 registers and one CTA per SM)
// SB_ZINV_MINB, SB_ZFWD_MINB: the same for the FP32 variants of the long
// transforms (N >= 288).  Four CTAs per SM (z-inverse 62 -> 55 registers,
// z-forward 94 -> 52, no spills) measured faster than the compiler's choice
// of three and two at 384x193x384: 0.547 -> 0.510 and 0.328 -> 0.269 ms;
// five measured slower, and at N = 96 the cap cost 2 %.
#ifndef SB_ZINV_MINB
#define SB_ZINV_MINB 4
#endif
#ifndef SB_ZFWD_MINB
#define SB_ZFWD_MINB 4
#endif
// SB_ZINV64_MINB: the FP64 variant (three CTAs of 288 threads at 72
// registers; four, at 56, measured 1.116 -> 1.148 ms at 384x193x384)
#ifndef SB_ZINV64_MINB
#define SB_ZINV64_MINB 3
#endif
template <class T, int KB, class S, int N = 0, int NT = 0>
__global__ void __launch_bounds__(NT > 0 ? NT : 256,
                                  (NT > 0 && sizeof(T) == 8) ? SB_ZINV64_MINB
                                                             : (NT > 0 && N >= 288 ? SB_ZINV_MINB : 0))
    k_zinv(const typename C2<S>::type* __restrict__ st, typename C2<T>::type* __restrict__ zb, Dims g,
           FFTPlan plan, const typename C2<T>::type* __restrict__ tw, const double* __restrict__ alfa,
           const double* __restrict__ beta, int drop_mean) {
  typedef typename C2<T>::type V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nzp = N > 0 ? N : g.nzp;
  const int nthr = NT > 0 ? NT : (int)blockDim.x;
  V* b0 = reinterpret_cast<V*>(smem_raw);
  V* b1 = b0 + (size_t)nzp * KB;
  const int y = g.y0 + blockIdx.y;
  const int kx0 = blockIdx.x * KB;
  const int nzh = g.nz / 2;
  const size_t slot = (size_t)g.nyp * g.NP;
  // fine-grid fields: 0 u, 1 v, 2 w, 3 omega_x, 4 omega_y, 5 omega_z
  const int src_slot[6] = {0, 1, 2, 3, -1, 4};
  typedef typename C2<S>::type SV;
  const SV* __restrict__ plane = st + (size_t)y * g.NP;  // this y-plane of slot 0
  for (int f = 0; f < 6; ++f) {
    const SV* __restrict__ src = plane + (size_t)(f == 4 ? 0 : src_slot[f]) * slot;
    if (SB_Z_PREFETCH && sizeof(T) == 8 && f + 1 < 6 && kx0 < g.nx2) {
      // field f + 1: its slot (omega_y: u and w) at the stored kz rows
      const SV* __restrict__ nsrc = plane + (size_t)(f + 1 == 4 ? 0 : src_slot[f + 1]) * slot + kx0;
      for (int iz = threadIdx.x; iz < g.nz; iz += nthr) {
        z_prefetch_l2(nsrc + (size_t)iz * g.nx2);
        if (f + 1 == 4) z_prefetch_l2(nsrc + 2 * slot + (size_t)iz * g.nx2);
      }
    }
    // element m (padded z index) of column b of field f
    auto load_elem = [&](int f, int m, int b) -> V {
      const int kx = kx0 + b;
      int iz = -1;
      if (m < nzh)
        iz = m;
      else if (m > nzp - nzh)
        iz = m - (nzp - g.nz);
      V val = V{(T)0, (T)0};
      if (iz >= 0 && kx < g.nx2 && !(drop_mean && iz == 0 && kx == 0)) {
        const int off = iz * g.nx2 + kx;
        if (f == 4) {
          const SV u = src[off];
          const SV w = src[2 * slot + off];
          const double a = alfa[kx], be = beta[iz];
          val = V{(T)(-be * (double)u.y + a * (double)w.y), (T)(be * (double)u.x - a * (double)w.x)};
        } else {
          const SV q = src[off];
          val = V{(T)q.x, (T)q.y};
        }
      }
      return val;
    };
    V* __restrict__ out = zb + ((size_t)f * g.nyp + y) * nzp * g.nx2;
    if constexpr (N > 0) {
      // the first pass reads the state, the last writes zb: shared memory
      // only between passes; FP32: the zero band of the padding (nz/2 <= m
      // <= nzp - nz/2, nzp = N = 3 nz / 2) is not loaded (FP64 measured 1 %
      // slower with it)
      cfft_io<T, KB, N, 1, NT, 0, sizeof(T) == 4>([&](int m, int b) { return load_elem(f, m, b); },
                               [&](int m, int b, V v) {
                                 if (kx0 + b < g.nx2) out[(size_t)m * g.nx2 + kx0 + b] = v;
                               },
                               b0, b1, tw, threadIdx.x);
    } else {
      for (int t = threadIdx.x; t < nzp * KB; t += nthr) {
        const int m = t / KB;
        b0[t] = load_elem(f, m, t - m * KB);
      }
      __syncthreads();
      V* res = fft_any<T, KB, N, NT, 1>(b0, b1, plan, tw);
      for (int t = threadIdx.x; t < nzp * KB; t += nthr) {
        const int m = t / KB;
        const int kx = kx0 + (t - m * KB);
        if (kx < g.nx2) out[(size_t)m * g.nx2 + kx] = res[t];
      }
    }
    __syncthreads();
  }
}

// CFL accumulator: non-negative doubles order like their bit patterns.
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// H -= lambda (u - U_b) at x point j of plane y.  u, v, w are the velocities
// the products used; um, wm the plane means they leave out (the mixed path's
// perturbation form, 0 on the FP64 path), which enter as U - U_b in FP64 so
// that no O(1) difference is rounded to FP32.  FP64 path: u + (-U_b) is the
// reference's u - U_b exactly.
template <class T>
__device__ __forceinline__ void fringe_apply(const Fringe& fr, int j, int y, int nyp, int n, T u, T v, T w,
                                             double um, double wm, T& h1, T& h2, T& h3) {
  const double lm = fr.lam[j];
  if (lm == 0.0) return;
  const size_t cs = (size_t)nyp * n;  // one component of the base flow
  const double* b = fr.base + (size_t)y * n + j;
  const T l = (T)lm;
  h1 = h1 - l * (u + (T)(um - b[0]));
  h2 = h2 - l * (v + (T)(0.0 - b[cs]));
  h3 = h3 - l * (w + (T)(wm - b[2 * cs]));
}

// N > 0: the x length g.nxp is N (compile-time plan, NT threads per CTA).
// SB_XPASS_MINB: resident CTAs per SM the FP32 fixed-length variant's
// register budget is sized for (0: the compiler's choice, three CTAs of 448
// threads at 40 registers; four at 32 registers measured the same)
#ifndef SB_XPASS_MINB
#define SB_XPASS_MINB 0
#endif
// SB_XPASS64_MINB: the same for the FP64 fixed-length variant (0: the
// compiler's choice, four CTAs of 224 threads at 66 registers; five, at 56
// registers and a 20-byte spill, measured 2.24 -> 2.34 ms at 384x193x384)
#ifndef SB_XPASS64_MINB
#define SB_XPASS64_MINB 0
#endif
template <class T, int RB, int N = 0, int NT = 0>
__global__ void __launch_bounds__(NT > 0 ? NT : 256,
                                  NT > 0 ? (sizeof(T) == 4 ? SB_XPASS_MINB : SB_XPASS64_MINB) : 0)
    k_xpass(const typename C2<T>::type* __restrict__ zb, typename C2<T>::type* __restrict__ xb, Dims g,
            FFTPlan plan, const typename C2<T>::type* __restrict__ tw, const double* __restrict__ dyi, double dxi,
            double dzi, double rot, unsigned long long* __restrict__ cfl_bits, const double* __restrict__ mean,
            Fringe fr) {
  typedef typename C2<T>::type V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int B = 3 * RB;
  const int n = N > 0 ? N : g.nxp;
  const int nthr = NT > 0 ? NT : (int)blockDim.x;
  V* bA = reinterpret_cast<V*>(smem_raw);
  V* bB = bA + (size_t)n * B;
  const int y = g.y0 + blockIdx.y;
  const int m0 = blockIdx.x * RB;
  // Hermitian completion of two half spectra into one complex spectrum:
  // element k of column c = 3 r + q (row m0 + r, fields 2q and 2q+1)
  const size_t fstride = (size_t)g.nyp * g.nzp * g.nx2;                   // one field of zb
  const V* __restrict__ zrow = zb + ((size_t)y * g.nzp + m0) * g.nx2;  // row m0 of field 0
  auto herm = [&](int k, int c) -> V {
    const int r = c / 3, q = c - 3 * r;
    V z = V{(T)0, (T)0};
    if (m0 + r < g.nzp) {
      const V* __restrict__ p0 = zrow + (size_t)(2 * q) * fstride + r * g.nx2;
      const V* __restrict__ p1 = p0 + fstride;
      if (k == 0) {
        z = V{p0[0].x, p1[0].x};
      } else if (k < g.nx2) {
        const V a = p0[k], b = p1[k];
        z = V{a.x - b.y, a.y + b.x};
      } else if (k > n - g.nx2) {
        const int kk = n - k;
        const V a = p0[kk], b = p1[kk];
        z = V{a.x + b.y, b.x - a.y};
      }
    }
    return z;
  };
  V* res;
  if constexpr (N > 0) {
    // the first inverse pass reads the spectra itself, except the zero band
    // nx/2 <= k <= nxp - nx/2 of the padding (nxp = N = 3 nx / 2)
    res = cfft_ld<T, B, N, 1, NT, true>(herm, bA, bB, tw, threadIdx.x);
  } else {
    for (int t = threadIdx.x; t < n * B; t += nthr) {
      const int k = t / B;
      bA[t] = herm(k, t - k * B);
    }
    __syncthreads();
    res = fft_any<T, B, N, NT, 1>(bA, bB, plan, tw);
  }
  V* oth = (res == bA) ? bB : bA;
  // products in physical space, H into (H1 + i H2) per row and, for an even
  // number of rows, the H3 of rows 2q and 2q+1 paired as H3 + i H3' (one
  // complex FFT for two real rows); a single row keeps (H3 + 0i).  CFL.
  constexpr int B2 = (RB % 2 == 0) ? RB + RB / 2 : 2 * RB;
  // Plane means (mixed path): u, w, omega_x, omega_z are perturbations; the
  // means U, W, Omega_x, Omega_z + 2 rot enter term by term so no product of
  // two O(1) means is rounded here (their W Omega_x - U Omega_z goes to the
  // kx = kz = 0 mode in FP64, in k_zfwd).  V = Omega_y = 0.  The CFL number
  // is formed in T (FP64 path: exactly the reference's sum).
  T U = (T)0, W = (T)0, Ox = (T)0, Oz = (T)0;
  if (mean != nullptr) {
    U = (T)mean[0 * g.nyp + y];
    W = (T)mean[1 * g.nyp + y];
    Ox = (T)mean[2 * g.nyp + y];
    Oz = (T)(mean[3 * g.nyp + y] + 2.0 * rot);
  }
  const T r2 = (T)(2.0 * rot);
  const T cx = (T)dxi, cy = (T)dyi[y], cz = (T)dzi;
  T cmaxt = (T)0;
  for (int t = threadIdx.x; t < n * RB; t += nthr) {
    const int j = t / RB;
    const int r = t - j * RB;
    const V z0 = res[j * B + 3 * r + 0];
    const V z1 = res[j * B + 3 * r + 1];
    const V z2 = res[j * B + 3 * r + 2];
    const T u = z0.x, v = z0.y, w = z1.x, ox = z1.y, oy = z2.x, oz = z2.y;
    T h1, h2, h3;
    if (mean == nullptr) {
      h1 = v * (oz + r2) - w * oy;
      h2 = w * ox - u * (oz + r2);
      h3 = u * oy - v * ox;
    } else {
      h1 = v * Oz + (v * oz - (W + w) * oy);
      h2 = (W * ox + w * Ox - U * oz - u * Oz) + (w * ox - u * oz);
      h3 = U * oy - v * Ox + (u * oy - v * ox);
    }
    // fringe on the total velocity (no plane means on the FP64 path)
    if (fr.lam != nullptr)
      fringe_apply<T>(fr, j, y, g.nyp, n, u, v, w, mean != nullptr ? mean[0 * g.nyp + y] : 0.0,
                      mean != nullptr ? mean[1 * g.nyp + y] : 0.0, h1, h2, h3);
    if constexpr (RB % 2 == 0) {
      oth[j * B2 + r] = V{h1, h2};
      T* h3p = reinterpret_cast<T*>(&oth[j * B2 + RB + r / 2]);
      h3p[r & 1] = h3;
    } else {
      oth[j * B2 + 2 * r + 0] = V{h1, h2};
      oth[j * B2 + 2 * r + 1] = V{h3, (T)0};
    }
    if (m0 + r < g.nzp) {
      const T cl = fabs(u + U) * cx + fabs(v) * cy + fabs(w + W) * cz;
      cmaxt = fmax(cmaxt, cl);
    }
  }
  double cmax = (double)cmaxt;
  __syncthreads();
  // (the band nx/2 <= k <= nxp - nx/2 of the spectra, which the loop below
  // never reads, is not written)
  V* fres = fft_any<T, B2, N, NT, -1, true>(oth, res, plan, tw);
  for (int t = threadIdx.x; t < g.nx2 * RB; t += nthr) {
    const int k = t / RB;
    const int r = t - k * RB;
    const int m = m0 + r;
    if (m >= g.nzp) continue;
    const int kk = (n - k) % n;
    V a, b, h3;
    if constexpr (RB % 2 == 0) {
      a = fres[k * B2 + r];
      b = fres[kk * B2 + r];
      // spectra of the real and imaginary rows of the paired H3 column
      const V c3 = fres[k * B2 + RB + r / 2], d3 = fres[kk * B2 + RB + r / 2];
      h3 = (r & 1) ? V{(c3.y + d3.y) * (T)0.5, (d3.x - c3.x) * (T)0.5}
                   : V{(c3.x + d3.x) * (T)0.5, (c3.y - d3.y) * (T)0.5};
    } else {
      a = fres[k * B2 + 2 * r];
      b = fres[kk * B2 + 2 * r];
      h3 = fres[k * B2 + 2 * r + 1];
    }
    const V h1 = V{(a.x + b.x) * (T)0.5, (a.y - b.y) * (T)0.5};
    const V h2 = V{(a.y + b.y) * (T)0.5, (b.x - a.x) * (T)0.5};
    V* __restrict__ o = xb + ((size_t)y * g.nzp + m0) * g.nx2 + r * g.nx2 + k;
    o[0] = h1;
    o[fstride] = h2;
    o[2 * fstride] = h3;
  }
  // block max of the CFL number
  for (int off = 16; off > 0; off >>= 1) cmax = fmax(cmax, __shfl_xor_sync(0xffffffffu, cmax, off));
  __shared__ double wmax[32];
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = cmax;
  __syncthreads();
  if (threadIdx.x == 0 && cfl_bits != nullptr) {
    double mx = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) mx = fmax(mx, wmax[i]);
    atomic_max_nonneg(cfl_bits, mx);
  }
}

// mean != nullptr: add nxp*nzp*(W Omega_x - U (Omega_z + 2 rot)) to the
// kx = kz = 0 mode of H2 in FP64 (the mean-mean product left out by k_xpass).
// FP64 z-forward: three CTAs per SM (102 -> 72 registers, an 8-byte spill)
// measured 0.710 -> 0.633 ms at 384x193x384 against the compiler's two
#ifndef SB_ZFWD64_MINB
#define SB_ZFWD64_MINB 3
#endif
template <class T, int KB, class S, int N = 0, int NT = 0>
__global__ void __launch_bounds__(NT > 0 ? NT : 256,
                                  NT > 0 ? (sizeof(T) == 4 ? (N >= 288 ? SB_ZFWD_MINB : 0) : SB_ZFWD64_MINB) : 0)
    k_zfwd(const typename C2<T>::type* __restrict__ xb, typename C2<S>::type* __restrict__ st, Dims g,
           FFTPlan plan, const typename C2<T>::type* __restrict__ tw, const double* __restrict__ mean, double rot) {
  typedef typename C2<T>::type V;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nzp = N > 0 ? N : g.nzp;
  const int nthr = NT > 0 ? NT : (int)blockDim.x;
  V* b0 = reinterpret_cast<V*>(smem_raw);
  V* b1 = b0 + (size_t)nzp * KB;
  const int y = g.y0 + blockIdx.y;
  const int kx0 = blockIdx.x * KB;
  const int nzh = g.nz / 2;
  const size_t fs = (size_t)g.nyp * nzp * g.nx2;
  const size_t slot = (size_t)g.nyp * g.NP;
  for (int f = 0; f < 3; ++f) {
    const V* __restrict__ in = xb + f * fs + (size_t)y * nzp * g.nx2;
    if (SB_Z_PREFETCH && sizeof(T) == 8 && f + 1 < 3 && kx0 < g.nx2) {
      const V* __restrict__ nin = in + fs + kx0;  // field f + 1, this CTA's columns
      for (int m = threadIdx.x; m < nzp; m += nthr) z_prefetch_l2(nin + (size_t)m * g.nx2);
    }
    typename C2<S>::type* __restrict__ dst = st + f * slot + (size_t)y * g.NP;
    // mode iz of column b (padded index m) into state slot f; the kx = kz = 0
    // mode of H2 gets the mean-mean product in FP64
    auto store = [&](int iz, int b, V h) {
      const int kx = kx0 + b;
      double hx = (double)h.x, hy = (double)h.y;
      if (mean != nullptr && f == 1 && iz == 0 && kx == 0) {
        const double U = mean[0 * g.nyp + y], W = mean[1 * g.nyp + y];
        const double Ox = mean[2 * g.nyp + y], Oz = mean[3 * g.nyp + y] + 2.0 * rot;
        hx += (double)g.nxp * (double)g.nzp * (W * Ox - U * Oz);
      }
      dst[iz * g.nx2 + kx] = typename C2<S>::type{(S)hx, (S)hy};
    };
    if constexpr (N > 0) {
      cfft_io<T, KB, N, -1, NT, 0, false, true>(
          [&](int m, int b) { return (kx0 + b < g.nx2) ? in[(size_t)m * g.nx2 + kx0 + b] : V{(T)0, (T)0}; },
          [&](int m, int b, V v) {
            // keep the nz stored modes (truncation folded into the store)
            if (kx0 + b >= g.nx2) return;
            if (m < nzh)
              store(m, b, v);
            else if (m >= nzp - nzh)
              store(m - (nzp - g.nz), b, v);
          },
          b0, b1, tw, threadIdx.x);
    } else {
      for (int t = threadIdx.x; t < nzp * KB; t += nthr) {
        const int m = t / KB;
        const int kx = kx0 + (t - m * KB);
        b0[t] = (kx < g.nx2) ? in[(size_t)m * g.nx2 + kx] : V{(T)0, (T)0};
      }
      __syncthreads();
      V* res = fft_any<T, KB, N, NT, -1>(b0, b1, plan, tw);
      for (int t = threadIdx.x; t < g.nz * KB; t += nthr) {
        const int iz = t / KB;
        const int b = t - iz * KB;
        if (kx0 + b >= g.nx2) continue;
        const int m = (iz < nzh) ? iz : iz + (nzp - g.nz);
        store(iz, b, res[m * KB + b]);
      }
    }
    __syncthreads();
  }
}

}  // namespace sb

namespace sb {
// Mean profiles U, W, Omega_x, Omega_z (the kx = kz = 0 coefficients of state
// slots 0, 2, 3, 4) into mean[4][nyp], read by the mixed-precision step 2.
template <class S>
__global__ void k_mean_profiles(const typename C2<S>::type* __restrict__ st, double* __restrict__ mean, Dims g) {
  const int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= g.nyp) return;
  const size_t slot = (size_t)g.nyp * g.NP;
  const int src[4] = {0, 2, 3, 4};
  for (int k = 0; k < 4; ++k) mean[k * g.nyp + y] = (double)st[src[k] * slot + (size_t)y * g.NP].x;
}
}  // namespace sb
