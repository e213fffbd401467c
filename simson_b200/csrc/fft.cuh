// Shared-memory Stockham FFT used by every transform of the step.
//
// A CTA transforms B columns of length n at once.  Columns are interleaved in
// shared memory (element i of column b at buf[i*B + b]) so that a warp reads
// consecutive columns of the same element: the layout the global loads of an
// xz-plane (z-FFT over kx columns) or of a y-pencil tile (Chebyshev transform
// over pencils) produce without any transpose.
//
// Each pass is one radix-R Stockham step (R in {2,3,4,5}, autosort, ping-pong
// between two buffers).  Twiddles come from a host-computed table
// tw[m] = exp(-2 pi i m / n); sign = -1 is the forward (analysis) transform,
// +1 the backward (synthesis) transform.  No normalisation is applied.
#pragma once
#include <type_traits>
#include <cuda_runtime.h>

#include <cmath>

#ifndef SB_HD
#define SB_HD __host__ __device__
#endif

namespace sb {

template <class T> struct C2;
template <> struct C2<double> { typedef double2 type; };
template <> struct C2<float> { typedef float2 type; };

template <class V> SB_HD __forceinline__ V cadd(V a, V b) { return V{a.x + b.x, a.y + b.y}; }
template <class V> SB_HD __forceinline__ V csub(V a, V b) { return V{a.x - b.x, a.y - b.y}; }
SB_HD __forceinline__ double fma_(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
SB_HD __forceinline__ float fma_(float a, float b, float c) {
#ifdef __CUDA_ARCH__
  return __fmaf_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
// complex product with explicit fused multiply-adds (the FFTs are not the
// parity-sensitive part of the step; the tau solves are built without FMA)
template <class V> SB_HD __forceinline__ V cmul(V a, V b) {
  return V{fma_(a.x, b.x, -a.y * b.y), fma_(a.x, b.y, a.y * b.x)};
}
template <class V> SB_HD __forceinline__ V cconj(V a) { return V{a.x, -a.y}; }
// multiply by i*s (s = +-1)
template <class V> SB_HD __forceinline__ V cmuli(V a, int s) {
  return s > 0 ? V{-a.y, a.x} : V{a.y, -a.x};
}

struct FFTPlan {
  int n;
  int npass;
  int radix[20];
  int ns[20];              // sub-transform length before the pass
  unsigned magic[20];      // ceil(2^32 / ns): j / ns == __umulhi(j, magic) for j*ns < 2^32
  int tstep[20];           // n / (ns * radix): twiddle stride of the pass
};

// cos and sin of 2*pi/5 and 4*pi/5 (the radix-5 butterfly)
#define SB_C5_1 0.30901699437494742410229341718281905886
#define SB_S5_1 0.95105651629515357211643933337938214340
#define SB_C5_2 (-0.80901699437494742410229341718281905886)
#define SB_S5_2 0.58778525229247312916870595463907276860
#define SB_S3 0.86602540378443864676372317075293618347
#define SB_R2 0.70710678118654752440084436210484903928
// cos and sin of 2*pi/9, 4*pi/9, 8*pi/9 (the radix-9 inner twiddles)
#define SB_C9_1 0.76604444311897803520239265055541667394
#define SB_S9_1 0.64278760968653932632264340990726343291
#define SB_C9_2 0.17364817766693034885171662676931479600
#define SB_S9_2 0.98480775301220805936674302458952301367
#define SB_C9_4 (-0.93969262078590838405410927732473146993)
#define SB_S9_4 0.34202014332566873304409961468225958076

template <class T, class V>
SB_HD __forceinline__ void dft3(V& a, V& b, V& c, int s) {
  V sum = cadd(b, c);
  V dif = csub(b, c);
  V m = V{a.x - (T)0.5 * sum.x, a.y - (T)0.5 * sum.y};
  V r = cmuli(V{(T)SB_S3 * dif.x, (T)SB_S3 * dif.y}, s);
  a = cadd(a, sum);
  b = cadd(m, r);
  c = csub(m, r);
}

// dft3 of (a, 0, c): the same operations as dft3 with b = 0 and the terms
// that add or subtract that zero left out (equal results up to the sign of
// an exact zero)
template <class T, class V>
SB_HD __forceinline__ void dft3_zmid(V& a, V& b, V& c, int s) {
  const V dif = V{-c.x, -c.y};
  const V m = V{a.x - (T)0.5 * c.x, a.y - (T)0.5 * c.y};
  const V r = cmuli(V{(T)SB_S3 * dif.x, (T)SB_S3 * dif.y}, s);
  a = cadd(a, c);
  b = cadd(m, r);
  c = csub(m, r);
}

template <class T, class V>
SB_HD __forceinline__ void dft4(V& a, V& b, V& c, V& d, int s) {
  V a0 = cadd(a, c), a1 = csub(a, c);
  V b0 = cadd(b, d), b1 = cmuli(csub(b, d), s);
  a = cadd(a0, b0);
  c = csub(a0, b0);
  b = cadd(a1, b1);
  d = csub(a1, b1);
}

// multiply by exp(s*i*2pi*k/8) for k = 1, 3 (k = 2 is cmuli)
template <class T, class V> SB_HD __forceinline__ V w8_1(V a, int s) {
  // (1 + s i)/sqrt2 * a
  return s > 0 ? V{(T)SB_R2 * (a.x - a.y), (T)SB_R2 * (a.x + a.y)} : V{(T)SB_R2 * (a.x + a.y), (T)SB_R2 * (a.y - a.x)};
}
template <class T, class V> SB_HD __forceinline__ V w8_3(V a, int s) {
  // (-1 + s i)/sqrt2 * a
  return s > 0 ? V{(T)SB_R2 * (-a.x - a.y), (T)SB_R2 * (a.x - a.y)} : V{(T)SB_R2 * (a.y - a.x), (T)SB_R2 * (-a.x - a.y)};
}

template <class T, class V>
SB_HD __forceinline__ void dft_small(V* v, int R, int s) {
  if (R == 8) {
    // radix-2 over stride 4, twiddles w8^k, then two radix-4 DFTs
    V e0 = cadd(v[0], v[4]), o0 = csub(v[0], v[4]);
    V e1 = cadd(v[1], v[5]), o1 = w8_1<T, V>(csub(v[1], v[5]), s);
    V e2 = cadd(v[2], v[6]), o2 = cmuli(csub(v[2], v[6]), s);
    V e3 = cadd(v[3], v[7]), o3 = w8_3<T, V>(csub(v[3], v[7]), s);
    dft4<T, V>(e0, e1, e2, e3, s);
    dft4<T, V>(o0, o1, o2, o3, s);
    v[0] = e0; v[2] = e1; v[4] = e2; v[6] = e3;
    v[1] = o0; v[3] = o1; v[5] = o2; v[7] = o3;
    return;
  }
  if (R == 6) {
    // radix-2 over stride 3 (w6^k twiddles), then two radix-3 DFTs
    V e0 = cadd(v[0], v[3]), o0 = csub(v[0], v[3]);
    V e1 = cadd(v[1], v[4]), d1 = csub(v[1], v[4]);
    V e2 = cadd(v[2], v[5]), d2 = csub(v[2], v[5]);
    // w6 = 1/2 + s i sqrt3/2 ; w6^2 = -1/2 + s i sqrt3/2
    V o1 = V{(T)0.5 * d1.x, (T)0.5 * d1.y};
    o1 = cadd(o1, cmuli(V{(T)SB_S3 * d1.x, (T)SB_S3 * d1.y}, s));
    V o2 = V{(T)-0.5 * d2.x, (T)-0.5 * d2.y};
    o2 = cadd(o2, cmuli(V{(T)SB_S3 * d2.x, (T)SB_S3 * d2.y}, s));
    dft3<T, V>(e0, e1, e2, s);
    dft3<T, V>(o0, o1, o2, s);
    v[0] = e0; v[2] = e1; v[4] = e2;
    v[1] = o0; v[3] = o1; v[5] = o2;
    return;
  }
  if (R == 9) {
    // radix-3 over stride 3, inner twiddles w9^(k*m), radix-3 again
    V a0 = v[0], a1 = v[3], a2 = v[6];
    V b0 = v[1], b1 = v[4], b2 = v[7];
    V c0 = v[2], c1 = v[5], c2 = v[8];
    dft3<T, V>(a0, a1, a2, s);
    dft3<T, V>(b0, b1, b2, s);
    dft3<T, V>(c0, c1, c2, s);
    const V w1 = V{(T)SB_C9_1, (T)(s * SB_S9_1)}, w2 = V{(T)SB_C9_2, (T)(s * SB_S9_2)};
    const V w4 = V{(T)SB_C9_4, (T)(s * SB_S9_4)};
    b1 = cmul(b1, w1);
    b2 = cmul(b2, w2);
    c1 = cmul(c1, w2);
    c2 = cmul(c2, w4);
    dft3<T, V>(a0, b0, c0, s);
    dft3<T, V>(a1, b1, c1, s);
    dft3<T, V>(a2, b2, c2, s);
    v[0] = a0; v[3] = b0; v[6] = c0;
    v[1] = a1; v[4] = b1; v[7] = c1;
    v[2] = a2; v[5] = b2; v[8] = c2;
    return;
  }
  if (R == 2) {
    V a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (R == 4) {
    V a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    V b0 = cadd(v[1], v[3]), b1 = cmuli(csub(v[1], v[3]), s);
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, b1);
    v[3] = csub(a1, b1);
  } else if (R == 3) {
    V sum = cadd(v[1], v[2]);
    V dif = csub(v[1], v[2]);
    V m = V{v[0].x - (T)0.5 * sum.x, v[0].y - (T)0.5 * sum.y};
    V r = cmuli(V{(T)SB_S3 * dif.x, (T)SB_S3 * dif.y}, s);
    v[0] = cadd(v[0], sum);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
  } else {  // R == 5
    V a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    V a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    V p1 = V{v[0].x + (T)SB_C5_1 * a1.x + (T)SB_C5_2 * a2.x, v[0].y + (T)SB_C5_1 * a1.y + (T)SB_C5_2 * a2.y};
    V p2 = V{v[0].x + (T)SB_C5_2 * a1.x + (T)SB_C5_1 * a2.x, v[0].y + (T)SB_C5_2 * a1.y + (T)SB_C5_1 * a2.y};
    V q1 = cmuli(V{(T)SB_S5_1 * b1.x + (T)SB_S5_2 * b2.x, (T)SB_S5_1 * b1.y + (T)SB_S5_2 * b2.y}, s);
    V q2 = cmuli(V{(T)SB_S5_2 * b1.x - (T)SB_S5_1 * b2.x, (T)SB_S5_2 * b1.y - (T)SB_S5_1 * b2.y}, s);
    v[0] = cadd(v[0], cadd(a1, a2));
    v[1] = cadd(p1, q1);
    v[4] = csub(p1, q1);
    v[2] = cadd(p2, q2);
    v[3] = csub(p2, q2);
  }
}

// dft_small with the inputs of mask ZM (bit r: v[r]) known to be zero: the
// radix-9 butterfly of a first pass whose middle third is the zero band
// skips the additions of those zeros; other radices use dft_small (the zeros
// are still not loaded)
template <class T, class V, unsigned ZM>
SB_HD __forceinline__ void dft_small_z(V* v, int R, int s) {
  if constexpr ((ZM & 0x38u) == 0x38u) {
    if (R == 9) {
      V a0 = v[0], a1 = v[3], a2 = v[6];
      V b0 = v[1], b1 = v[4], b2 = v[7];
      V c0 = v[2], c1 = v[5], c2 = v[8];
      dft3_zmid<T, V>(a0, a1, a2, s);
      dft3_zmid<T, V>(b0, b1, b2, s);
      dft3_zmid<T, V>(c0, c1, c2, s);
      const V w1 = V{(T)SB_C9_1, (T)(s * SB_S9_1)}, w2 = V{(T)SB_C9_2, (T)(s * SB_S9_2)};
      const V w4 = V{(T)SB_C9_4, (T)(s * SB_S9_4)};
      b1 = cmul(b1, w1);
      b2 = cmul(b2, w2);
      c1 = cmul(c1, w2);
      c2 = cmul(c2, w4);
      dft3<T, V>(a0, b0, c0, s);
      dft3<T, V>(a1, b1, c1, s);
      dft3<T, V>(a2, b2, c2, s);
      v[0] = a0; v[3] = b0; v[6] = c0;
      v[1] = a1; v[4] = b1; v[7] = c1;
      v[2] = a2; v[5] = b2; v[8] = c2;
      return;
    }
  }
  dft_small<T, V>(v, R, s);
}

// One Stockham pass: src -> dst, sub-transform length Ns -> Ns*R.  B (the
// number of interleaved columns) is a compile-time constant so the column
// index is a mask/shift; the only division left (by Ns) uses a precomputed
// reciprocal.  The twiddle exponent r*jm*tstep is always below n.
SB_HD __forceinline__ unsigned umulhi_(unsigned a, unsigned b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (unsigned)(((unsigned long long)a * b) >> 32);
#endif
}

// v[r] *= w^(r e), w = exp(S 2 pi i / n), from the table tw[m] = exp(-2 pi i m / n).
// Twiddle powers w^r, r = 1..R-1: two table loads (w, w^2) and products of
// depth <= 2 for the rest (a few ulp), in FP32 and, with SB_TW_PRODUCTS64, in
// FP64 too: the FP64 transforms were stalled on the R - 1 table loads per
// butterfly (x pass 2.25 -> 1.91 ms, z-inverse 1.02 -> 0.96, z-forward 0.55 ->
// 0.51 at 384x193x384; the parity gates against the reference unchanged)
#ifndef SB_TW_PRODUCTS64
#define SB_TW_PRODUCTS64 1
#endif
template <class T, int R, int S>
SB_HD __forceinline__ void twiddle(typename C2<T>::type* v, const typename C2<T>::type* __restrict__ tw, int e) {
  typedef typename C2<T>::type V;
  if constexpr (std::is_same<T, float>::value || SB_TW_PRODUCTS64) {
    // two table loads, the other powers by products of depth <= 2 (w^k for
    // k <= 8 from w, w^2: a few ulp), fewer load-pipe requests
    V w[9];
    w[1] = tw[e];
    w[2] = tw[2 * e];
    if (S > 0) {
      w[1].y = -w[1].y;
      w[2].y = -w[2].y;
    }
    if (R > 3) {
      w[3] = cmul(w[1], w[2]);
      w[4] = cmul(w[2], w[2]);
    }
    if (R > 5) {
      w[5] = cmul(w[1], w[4]);
      w[6] = cmul(w[3], w[3]);
    }
    if (R > 7) {
      w[7] = cmul(w[3], w[4]);
      w[8] = cmul(w[4], w[4]);
    }
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
  } else {
#pragma unroll
    for (int r = 1; r < R; ++r) {
      V w = tw[r * e];
      if (S > 0) w.y = -w.y;
      v[r] = cmul(v[r], w);
    }
  }
}

// S: transform sign (compile time), so the twiddle conjugation and the
// +-i rotations of the small DFTs fold into the arithmetic.
template <class T, int B, int R, int S>
SB_HD __forceinline__ void stockham_pass(const typename C2<T>::type* __restrict__ src,
                                         typename C2<T>::type* __restrict__ dst, int n, int Ns, unsigned magic,
                                         int tstep, const typename C2<T>::type* __restrict__ tw, int t0,
                                         int tstride) {
  typedef typename C2<T>::type V;
  const int nb = n / R;
  for (int t = t0; t < nb * B; t += tstride) {
    const int j = t / B;
    const int b = t - j * B;
    const int jg = (Ns == 1) ? j : (int)umulhi_((unsigned)j, magic);
    const int jm = j - jg * Ns;
    V v[9];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * B + b];
    if (jm != 0) twiddle<T, R, S>(v, tw, jm * tstep);
    dft_small<T, V>(v, R, S);
    const int base = jg * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(base + r * Ns) * B + b] = v[r];
  }
}

// One pass of radix plan.radix[p]: work items t0, t0+tstride, ...
template <class T, int B, int S>
SB_HD __forceinline__ void fft_pass_s(const typename C2<T>::type* src, typename C2<T>::type* dst,
                                      const FFTPlan& plan, int p, const typename C2<T>::type* __restrict__ tw, int t0,
                                      int tstride) {
  const int R = plan.radix[p];
  const int Ns = plan.ns[p];
  const unsigned mg = plan.magic[p];
  const int ts = plan.tstep[p];
  if (R == 8)
    stockham_pass<T, B, 8, S>(src, dst, plan.n, Ns, mg, ts, tw, t0, tstride);
  else if (R == 9)
    stockham_pass<T, B, 9, S>(src, dst, plan.n, Ns, mg, ts, tw, t0, tstride);
  else if (R == 6)
    stockham_pass<T, B, 6, S>(src, dst, plan.n, Ns, mg, ts, tw, t0, tstride);
  else if (R == 4)
    stockham_pass<T, B, 4, S>(src, dst, plan.n, Ns, mg, ts, tw, t0, tstride);
  else if (R == 2)
    stockham_pass<T, B, 2, S>(src, dst, plan.n, Ns, mg, ts, tw, t0, tstride);
  else if (R == 3)
    stockham_pass<T, B, 3, S>(src, dst, plan.n, Ns, mg, ts, tw, t0, tstride);
  else
    stockham_pass<T, B, 5, S>(src, dst, plan.n, Ns, mg, ts, tw, t0, tstride);
}

template <class T, int B>
SB_HD __forceinline__ void fft_pass(const typename C2<T>::type* src, typename C2<T>::type* dst, const FFTPlan& plan,
                                    int p, const typename C2<T>::type* __restrict__ tw, int s, int t0, int tstride) {
  if (s > 0)
    fft_pass_s<T, B, 1>(src, dst, plan, p, tw, t0, tstride);
  else
    fft_pass_s<T, B, -1>(src, dst, plan, p, tw, t0, tstride);
}

// Full transform of the B interleaved columns held in buf0; buf1 is scratch.
// Returns the buffer holding the result.  Caller syncs before; the function
// ends with a barrier.
template <class T, int B, int S>
__device__ typename C2<T>::type* fft_columns_s(typename C2<T>::type* buf0, typename C2<T>::type* buf1,
                                              const FFTPlan& plan, const typename C2<T>::type* __restrict__ tw) {
  typename C2<T>::type* src = buf0;
  typename C2<T>::type* dst = buf1;
  for (int p = 0; p < plan.npass; ++p) {
    fft_pass_s<T, B, S>(src, dst, plan, p, tw, threadIdx.x, blockDim.x);
    __syncthreads();
    typename C2<T>::type* tmp = src;
    src = dst;
    dst = tmp;
  }
  return src;
}

template <class T, int B>
__device__ __forceinline__ typename C2<T>::type* fft_columns(typename C2<T>::type* buf0, typename C2<T>::type* buf1,
                                                            const FFTPlan& plan,
                                                            const typename C2<T>::type* __restrict__ tw, int s) {
  return (s > 0) ? fft_columns_s<T, B, 1>(buf0, buf1, plan, tw) : fft_columns_s<T, B, -1>(buf0, buf1, plan, tw);
}

// Radix plan of an n-point transform: 9s first (the odd stride of the first,
// unit-Ns pass spreads its shared-memory stores over the banks: measured
// 3-5 % faster x pass), then 8, 6, 4, 2, 3, 5 (384 = 8 8 6 stays as it was:
// 6 first measured slower for the Chebyshev transforms).
inline FFTPlan fft_make_plan(int n) {
  FFTPlan p{};
  p.n = n;
  int m = n, k = 0;
  const int order[7] = {9, 8, 6, 4, 2, 3, 5};
  for (int r : order)
    while (m % r == 0 && k < 20) {
      p.radix[k++] = r;
      m /= r;
    }
  p.npass = (m == 1) ? k : -1;
  int ns = 1;
  for (int i = 0; i < k; ++i) {
    p.ns[i] = ns;
    p.magic[i] = (ns == 1) ? 0u : (unsigned)((((unsigned long long)1 << 32) + ns - 1) / ns);
    p.tstep[i] = n / (ns * p.radix[i]);
    ns *= p.radix[i];
  }
  return p;
}

// ---------------------------------------------------------------------------
// Compile-time plans.  For the transform lengths of the production grids the
// length N, the radix sequence, every Ns and the thread count NT are template
// constants: the element addresses of a pass become one base register plus
// immediate offsets, the index divisions become multiplies by constants, and
// the work-item loop has a known trip count.  Same radix order, twiddles and
// butterflies as the runtime plan above.
// ---------------------------------------------------------------------------
struct CPlanData {
  int npass;
  int radix[12];
  int ns[12];
};

constexpr CPlanData cplan_make(int n) {
  CPlanData p{};
  int m = n, k = 0;
  const int order[7] = {9, 8, 6, 4, 2, 3, 5};
  for (int oi = 0; oi < 7; ++oi)
    while (m % order[oi] == 0 && k < 12) {
      p.radix[k++] = order[oi];
      m /= order[oi];
    }
  p.npass = (m == 1) ? k : -1;
  int ns = 1;
  for (int i = 0; i < k; ++i) {
    p.ns[i] = ns;
    ns *= p.radix[i];
  }
  return p;
}

// The 3/2 zero padding of the step-2 transforms (n = 3/2 of the stored
// modes): an inverse transform's input is zero on the band [n/3, 2n/3] of
// padded indices, a forward transform's output is dropped on [n/3, 2n/3).
// pad_zero_mask: bit r set when input block r of the first pass (indices
// [r n/R, (r+1) n/R)) lies in the zero band; pad_drop_mask: bit r set when
// output block r of the last pass (indices [r Ns, (r+1) Ns)) lies in the
// dropped band.
template <int N>
constexpr unsigned pad_zero_mask() {
  constexpr CPlanData p = cplan_make(N);
  const int R = p.radix[0], nb = N / R;
  unsigned m = 0;
  for (int r = 0; r < R; ++r)
    if (3 * r * nb >= N && 3 * ((r + 1) * nb - 1) <= 2 * N) m |= 1u << r;
  return m;
}
template <int N>
constexpr unsigned pad_drop_mask() {
  constexpr CPlanData p = cplan_make(N);
  const int R = p.radix[p.npass - 1], ns = p.ns[p.npass - 1];
  unsigned m = 0;
  for (int r = 0; r < R; ++r)
    if (3 * r * ns >= N && 3 * (r + 1) * ns <= 2 * N) m |= 1u << r;
  return m;
}

// largest number of butterflies of one column in any pass (n / smallest radix)
constexpr int cplan_max_nb(int n) {
  const CPlanData p = cplan_make(n);
  int mx = 0;
  for (int i = 0; i < p.npass; ++i) mx = (n / p.radix[i] > mx) ? n / p.radix[i] : mx;
  return mx;
}

// One radix-R pass of an N-point transform over B interleaved columns; work
// items t0, t0 + NT, ...
// DM: outputs of the blocks in the mask are not stored (pad_drop_mask).
template <class T, int B, int N, int R, int NS, int S, int NT, unsigned DM = 0>
SB_HD __forceinline__ void cpass(const typename C2<T>::type* __restrict__ src, typename C2<T>::type* __restrict__ dst,
                                 const typename C2<T>::type* __restrict__ tw, int t0) {
  typedef typename C2<T>::type V;
  constexpr int nb = N / R;
  constexpr int items = nb * B;
  constexpr int tstep = N / (NS * R);
  constexpr int iters = (items + NT - 1) / NT;
#pragma unroll
  for (int it = 0; it < iters; ++it) {
    const int t = t0 + it * NT;
    if (items % NT != 0 && t >= items) break;
    const unsigned j = (unsigned)t / B;
    const unsigned b = (unsigned)t - j * B;
    const unsigned jg = j / NS;
    const unsigned jm = j - jg * NS;
    V v[9];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[t + r * nb * B];
    if (NS > 1 && jm != 0) twiddle<T, R, S>(v, tw, (int)(jm * tstep));
    dft_small<T, V>(v, R, S);
    V* __restrict__ d = dst + (size_t)((jg * NS * R + jm) * B + b);
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (!(DM & (1u << r))) d[r * NS * B] = v[r];
  }
}

// All passes of the N-point transform of the B columns in src (dst is
// scratch); returns the buffer holding the result.  On the device every pass
// ends with a barrier (the caller syncs before the first).
// DOUT: the output band that pad_drop_mask names is left unwritten (the
// caller reads only the kept modes).
template <class T, int B, int N, int S, int NT, int P = 0, bool DOUT = false>
SB_HD __forceinline__ typename C2<T>::type* cfft(typename C2<T>::type* src, typename C2<T>::type* dst,
                                                 const typename C2<T>::type* __restrict__ tw, int t0) {
  constexpr CPlanData pl = cplan_make(N);
  static_assert(pl.npass > 0, "transform length must factor into 2, 3, 5");
  if constexpr (P >= pl.npass) {
    return src;
  } else {
    constexpr unsigned dm = (DOUT && P == pl.npass - 1) ? pad_drop_mask<N>() : 0u;
    cpass<T, B, N, pl.radix[P], pl.ns[P], S, NT, dm>(src, dst, tw, t0);
#ifdef __CUDA_ARCH__
    __syncthreads();
#endif
    return cfft<T, B, N, S, NT, P + 1, DOUT>(dst, src, tw, t0);
  }
}

// One pass with accessors instead of shared-memory buffers: ld(m, b) returns
// element m of column b of the pass input, st(k, b, v) stores element k of
// column b of its output.  The first pass of cfft_io reads the global arrays
// through ld and its last pass writes them through st, so the data crosses
// shared memory only between passes.
// ZM: inputs of the blocks in the mask are zero and not loaded
// (pad_zero_mask, first pass); DM: outputs of the blocks in the mask are not
// stored (pad_drop_mask, last pass).
template <class T, int B, int N, int R, int NS, int S, int NT, unsigned ZM = 0, unsigned DM = 0, class Ld,
          class St>
SB_HD __forceinline__ void cpass_io(Ld ld, St st, const typename C2<T>::type* __restrict__ tw, int t0) {
  typedef typename C2<T>::type V;
  constexpr int nb = N / R;
  constexpr int items = nb * B;
  constexpr int tstep = N / (NS * R);
  constexpr int iters = (items + NT - 1) / NT;
#pragma unroll
  for (int it = 0; it < iters; ++it) {
    const int t = t0 + it * NT;
    if (items % NT != 0 && t >= items) break;
    const unsigned j = (unsigned)t / B;
    const unsigned b = (unsigned)t - j * B;
    const unsigned jg = j / NS;
    const unsigned jm = j - jg * NS;
    V v[9];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = (ZM & (1u << r)) ? V{(T)0, (T)0} : ld((int)(j + r * nb), (int)b);
    if (NS > 1 && jm != 0) twiddle<T, R, S>(v, tw, (int)(jm * tstep));
    dft_small_z<T, V, ZM>(v, R, S);
    const int k0 = (int)(jg * NS * R + jm);
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (!(DM & (1u << r))) st(k0 + r * NS, (int)b, v[r]);
  }
}

template <class T, int B>
struct SmemLd {
  const typename C2<T>::type* __restrict__ p;
  SB_HD __forceinline__ typename C2<T>::type operator()(int m, int b) const { return p[m * B + b]; }
};
template <class T, int B>
struct SmemSt {
  typename C2<T>::type* __restrict__ p;
  SB_HD __forceinline__ void operator()(int k, int b, typename C2<T>::type v) const { p[k * B + b] = v; }
};

// N-point transform of B columns from ld to st (at least two passes);
// buf0/buf1 hold the intermediate passes.  The caller syncs before reusing
// the buffers.
// ZIN: the input is zero on the band of pad_zero_mask (never loaded); DOUT:
// st is never called on the band of pad_drop_mask.
template <class T, int B, int N, int S, int NT, int P = 0, bool ZIN = false, bool DOUT = false, class Ld,
          class St>
SB_HD __forceinline__ void cfft_io(Ld ld, St st, typename C2<T>::type* buf0, typename C2<T>::type* buf1,
                                   const typename C2<T>::type* __restrict__ tw, int t0) {
  constexpr CPlanData pl = cplan_make(N);
  static_assert(pl.npass >= 2, "cfft_io needs at least two passes");
  if constexpr (P == 0) {
    cpass_io<T, B, N, pl.radix[0], pl.ns[0], S, NT, ZIN ? pad_zero_mask<N>() : 0u>(ld, SmemSt<T, B>{buf0}, tw,
                                                                                  t0);
#ifdef __CUDA_ARCH__
    __syncthreads();
#endif
    cfft_io<T, B, N, S, NT, 1, ZIN, DOUT>(ld, st, buf0, buf1, tw, t0);
  } else if constexpr (P == pl.npass - 1) {
    cpass_io<T, B, N, pl.radix[P], pl.ns[P], S, NT, 0u, DOUT ? pad_drop_mask<N>() : 0u>(SmemLd<T, B>{buf0}, st,
                                                                                       tw, t0);
  } else {
    cpass_io<T, B, N, pl.radix[P], pl.ns[P], S, NT>(SmemLd<T, B>{buf0}, SmemSt<T, B>{buf1}, tw, t0);
#ifdef __CUDA_ARCH__
    __syncthreads();
#endif
    cfft_io<T, B, N, S, NT, P + 1, ZIN, DOUT>(ld, st, buf1, buf0, tw, t0);
  }
}

// First pass from ld, the others in shared memory; returns the buffer that
// holds the result (ends with a barrier on the device).
template <class T, int B, int N, int S, int NT, bool ZIN = false, class Ld>
SB_HD __forceinline__ typename C2<T>::type* cfft_ld(Ld ld, typename C2<T>::type* buf0, typename C2<T>::type* buf1,
                                                    const typename C2<T>::type* __restrict__ tw, int t0) {
  constexpr CPlanData pl = cplan_make(N);
  cpass_io<T, B, N, pl.radix[0], pl.ns[0], S, NT, ZIN ? pad_zero_mask<N>() : 0u>(ld, SmemSt<T, B>{buf0}, tw, t0);
#ifdef __CUDA_ARCH__
  __syncthreads();
#endif
  return cfft<T, B, N, S, NT, 1>(buf0, buf1, tw, t0);
}

// runtime plan (N == 0) or compile-time plan, same interface (DOUT: as cfft,
// compile-time plans only)
template <class T, int B, int N, int NT, int S, bool DOUT = false>
__device__ __forceinline__ typename C2<T>::type* fft_any(typename C2<T>::type* buf0, typename C2<T>::type* buf1,
                                                        const FFTPlan& plan,
                                                        const typename C2<T>::type* __restrict__ tw) {
  if constexpr (N == 0)
    return fft_columns_s<T, B, S>(buf0, buf1, plan, tw);
  else
    return cfft<T, B, N, S, NT, 0, DOUT>(buf0, buf1, tw, threadIdx.x);
}

}  // namespace sb
