// Mixed-precision step kernels (declared in mixed.h), compiled with
// -fmad=true: FP32 transforms and products of step 2, and the pencil,
// homogeneous-solution and mean-flow kernels of step 3 with FP32 storage.
#include "mixed.h"
#include "step2_launch.cuh"
#include "pencil_warp.cuh"

namespace sb {

void mixed_mean_profiles(cudaStream_t s, const float2* stf, double* meanp, const Dims& g) {
  k_mean_profiles<float><<<(g.nyp + 127) / 128, 128, 0, s>>>(stf, meanp, g);
}

void mixed_zinv(cudaStream_t s, dim3 grid, size_t smem, const float2* stf, float2* zb, const Dims& g,
                const FFTPlan& plan, const float2* tw, const double* alfa, const double* beta) {
  launch_zinv<float, MIXED_KB, float>(grid, smem, s, stf, zb, g, plan, tw, alfa, beta, 1);
}

void mixed_xpass(cudaStream_t s, dim3 grid, size_t smem, const float2* zb, float2* xb, const Dims& g,
                 const FFTPlan& plan, const float2* tw, const double* dyi, double dxi, double dzi, double rot,
                 unsigned long long* cfl, const double* meanp, Fringe fr) {
  launch_xpass<float, MIXED_RB, SB_FFT_THREADS>(grid, smem, s, zb, xb, g, plan, tw, dyi, dxi, dzi, rot, cfl, meanp,
                                                fr);
}

void mixed_zfwd(cudaStream_t s, dim3 grid, size_t smem, const float2* xb, float2* stf, const Dims& g,
                const FFTPlan& plan, const float2* tw, const double* meanp, double rot) {
  launch_zfwd<float, MIXED_KB, float>(grid, smem, s, xb, stf, g, plan, tw, meanp, rot);
}

void mixed_pencil_hom(cudaStream_t s, const PencilBufs& B, const Dims& g, const double* alfa, const double* beta,
                      double re, double anbn, double* vh, double* hs, double* cf) {
  k_pencil_hom<double, float><<<(g.p1 - g.p0 + 127) / 128, 128, 0, s>>>(B, g, alfa, beta, re, anbn, vh, hs, cf);
}

void mixed_pencil(cudaStream_t s, const PencilBufs& B, const Dims& g, const double* alfa, const double* beta,
                  double re, RKc rk, const double* vh, const double* hs, double* cf) {
  k_pencil<float2, double, float><<<(g.p1 - g.p0 + 127) / 128, 128, 0, s>>>(B, g, alfa, beta, re, rk, vh, hs, cf);
}

bool mixed_pencil_warp(cudaStream_t s, const PencilBufs& B, const Dims& g, const double* alfa, const double* beta,
                       double re, RKc rk) {
  return launch_pencil_warp<float2, float>(s, B, g, alfa, beta, re, rk);
}

void mixed_mean(cudaStream_t s, const MeanArgs& M, const Dims& g, double re, RKc rk) {
  k_mean<float2><<<1, 32, 0, s>>>(M, g, re, rk);
}

}  // namespace sb
