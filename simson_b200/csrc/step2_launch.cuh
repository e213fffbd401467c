// Launch helpers of the step-2 kernels: transform lengths with compile-time
// plans get their own instantiations (fixed_threads threads per CTA), any
// other length the runtime plan.  Shared by the FP64 unit (simson.cu) and the
// mixed-precision unit (mixed.cu), each instantiating its own types.
#pragma once
#include <cuda_runtime.h>

#include "fft.cuh"
#include "layout.cuh"
#include "step2.cuh"

namespace sb {

// threads per CTA of the runtime-plan FFT kernels
constexpr int SB_FFT_THREADS = 256;

// Transform lengths with compile-time FFT plans (fft.cuh cfft): the
// production grid's 576 (3/2 x 384) and the test, LES and channel grids' 3/2
// lengths; any other length takes the runtime plan.
#define SB_FIXED_LENGTHS(X) X(72) X(96) X(240) X(288) X(576)

// threads per CTA for B columns of an N-point compile-time transform: one
// butterfly per thread in the widest pass (halved while above 512), a
// multiple of 32
constexpr int fixed_threads(int n, int b) {
  int items = cplan_max_nb(n) * b;
  while (items > 512) items = (items + 1) / 2;
  return ((items + 31) / 32) * 32;
}

template <class T, int KB, class S, int N, int NT>
inline void zinv_n(dim3 grid, size_t smem, cudaStream_t st, const typename C2<S>::type* in,
                   typename C2<T>::type* zb, const Dims& g, const FFTPlan& plan, const typename C2<T>::type* tw,
                   const double* alfa, const double* beta, int drop) {
  cudaFuncSetAttribute(k_zinv<T, KB, S, N, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_zinv<T, KB, S, N, NT><<<grid, NT, smem, st>>>(in, zb, g, plan, tw, alfa, beta, drop);
}
template <class T, int KB, class S>
inline void launch_zinv(dim3 grid, size_t smem, cudaStream_t st, const typename C2<S>::type* in,
                        typename C2<T>::type* zb, const Dims& g, const FFTPlan& plan,
                        const typename C2<T>::type* tw, const double* alfa, const double* beta, int drop) {
  switch (g.nzp) {
#define SB_CASE(n)                                                                                 \
  case n:                                                                                          \
    zinv_n<T, KB, S, n, fixed_threads(n, KB)>(grid, smem, st, in, zb, g, plan, tw, alfa, beta, drop); \
    return;
    SB_FIXED_LENGTHS(SB_CASE)
#undef SB_CASE
    default:
      zinv_n<T, KB, S, 0, SB_FFT_THREADS>(grid, smem, st, in, zb, g, plan, tw, alfa, beta, drop);
  }
}

template <class T, int KB, class S, int N, int NT>
inline void zfwd_n(dim3 grid, size_t smem, cudaStream_t st, const typename C2<T>::type* xb,
                   typename C2<S>::type* out, const Dims& g, const FFTPlan& plan, const typename C2<T>::type* tw,
                   const double* mean, double rot) {
  cudaFuncSetAttribute(k_zfwd<T, KB, S, N, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_zfwd<T, KB, S, N, NT><<<grid, NT, smem, st>>>(xb, out, g, plan, tw, mean, rot);
}
template <class T, int KB, class S>
inline void launch_zfwd(dim3 grid, size_t smem, cudaStream_t st, const typename C2<T>::type* xb,
                        typename C2<S>::type* out, const Dims& g, const FFTPlan& plan,
                        const typename C2<T>::type* tw, const double* mean, double rot) {
  switch (g.nzp) {
#define SB_CASE(n)                                                                          \
  case n:                                                                                   \
    zfwd_n<T, KB, S, n, fixed_threads(n, KB)>(grid, smem, st, xb, out, g, plan, tw, mean, rot); \
    return;
    SB_FIXED_LENGTHS(SB_CASE)
#undef SB_CASE
    default:
      zfwd_n<T, KB, S, 0, SB_FFT_THREADS>(grid, smem, st, xb, out, g, plan, tw, mean, rot);
  }
}

template <class T, int RB, int N, int NT>
inline void xpass_n(dim3 grid, size_t smem, cudaStream_t st, const typename C2<T>::type* zb,
                    typename C2<T>::type* xb, const Dims& g, const FFTPlan& plan, const typename C2<T>::type* tw,
                    const double* dyi, double dxi, double dzi, double rot, unsigned long long* cfl,
                    const double* mean, Fringe fr) {
  cudaFuncSetAttribute(k_xpass<T, RB, N, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
#ifdef SB_XPASS_CARVEOUT
  cudaFuncSetAttribute(k_xpass<T, RB, N, NT>, cudaFuncAttributePreferredSharedMemoryCarveout, SB_XPASS_CARVEOUT);
#endif
  k_xpass<T, RB, N, NT><<<grid, NT, smem, st>>>(zb, xb, g, plan, tw, dyi, dxi, dzi, rot, cfl, mean, fr);
}
template <class T, int RB, int NT0>
inline void launch_xpass(dim3 grid, size_t smem, cudaStream_t st, const typename C2<T>::type* zb,
                         typename C2<T>::type* xb, const Dims& g, const FFTPlan& plan,
                         const typename C2<T>::type* tw, const double* dyi, double dxi, double dzi, double rot,
                         unsigned long long* cfl, const double* mean, Fringe fr) {
  switch (g.nxp) {
#define SB_CASE(n)                                                                                        \
  case n:                                                                                                 \
    xpass_n<T, RB, n, fixed_threads(n, 3 * RB)>(grid, smem, st, zb, xb, g, plan, tw, dyi, dxi, dzi, rot, cfl, \
                                                mean, fr);                                                \
    return;
    SB_FIXED_LENGTHS(SB_CASE)
#undef SB_CASE
    default:
      xpass_n<T, RB, 0, NT0>(grid, smem, st, zb, xb, g, plan, tw, dyi, dxi, dzi, rot, cfl, mean, fr);
  }
}

}  // namespace sb
