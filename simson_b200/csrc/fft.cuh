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
#include <cuda_runtime.h>

namespace sb {

template <class T> struct C2;
template <> struct C2<double> { typedef double2 type; };
template <> struct C2<float> { typedef float2 type; };

template <class V> __device__ __forceinline__ V cadd(V a, V b) { return V{a.x + b.x, a.y + b.y}; }
template <class V> __device__ __forceinline__ V csub(V a, V b) { return V{a.x - b.x, a.y - b.y}; }
template <class V> __device__ __forceinline__ V cmul(V a, V b) {
  return V{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <class V> __device__ __forceinline__ V cconj(V a) { return V{a.x, -a.y}; }
// multiply by i*s (s = +-1)
template <class V> __device__ __forceinline__ V cmuli(V a, int s) {
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

template <class T, class V>
__device__ __forceinline__ void dft_small(V* v, int R, int s) {
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

// One Stockham pass: src -> dst, sub-transform length Ns -> Ns*R.  B (the
// number of interleaved columns) is a compile-time constant so the column
// index is a mask/shift; the only division left (by Ns) uses a precomputed
// reciprocal.  The twiddle exponent r*jm*tstep is always below n.
template <class T, int B, int R>
__device__ __forceinline__ void stockham_pass(const typename C2<T>::type* __restrict__ src,
                                              typename C2<T>::type* __restrict__ dst, int n, int Ns,
                                              unsigned magic, int tstep,
                                              const typename C2<T>::type* __restrict__ tw, int s) {
  typedef typename C2<T>::type V;
  const int nb = n / R;
  for (int t = threadIdx.x; t < nb * B; t += blockDim.x) {
    const int j = t / B;
    const int b = t - j * B;
    const int jg = (Ns == 1) ? j : (int)__umulhi((unsigned)j, magic);
    const int jm = j - jg * Ns;
    V v[5];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * B + b];
    if (jm != 0) {
      const int e = jm * tstep;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        V w = tw[r * e];
        if (s > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dft_small<T, V>(v, R, s);
    const int base = jg * Ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(base + r * Ns) * B + b] = v[r];
  }
}

// Full transform of the B interleaved columns held in buf0; buf1 is scratch.
// Returns the buffer holding the result.  Caller syncs before; the function
// ends with a barrier.
template <class T, int B>
__device__ typename C2<T>::type* fft_columns(typename C2<T>::type* buf0, typename C2<T>::type* buf1,
                                            const FFTPlan& plan, const typename C2<T>::type* __restrict__ tw,
                                            int s) {
  typename C2<T>::type* src = buf0;
  typename C2<T>::type* dst = buf1;
  for (int p = 0; p < plan.npass; ++p) {
    const int R = plan.radix[p];
    const int Ns = plan.ns[p];
    if (R == 4)
      stockham_pass<T, B, 4>(src, dst, plan.n, Ns, plan.magic[p], plan.tstep[p], tw, s);
    else if (R == 2)
      stockham_pass<T, B, 2>(src, dst, plan.n, Ns, plan.magic[p], plan.tstep[p], tw, s);
    else if (R == 3)
      stockham_pass<T, B, 3>(src, dst, plan.n, Ns, plan.magic[p], plan.tstep[p], tw, s);
    else
      stockham_pass<T, B, 5>(src, dst, plan.n, Ns, plan.magic[p], plan.tstep[p], tw, s);
    __syncthreads();
    typename C2<T>::type* tmp = src;
    src = dst;
    dst = tmp;
  }
  return src;
}

}  // namespace sb
