// Launchers of the mixed-precision path's step kernels.  They live in their
// own translation unit (mixed.cu), built with fused multiply-add contraction:
// the mixed path is checked against the FP64 path at 1e-5, not bit for bit,
// while the FP64 unit (simson.cu) is built without contraction to stay at the
// reference's roundoff floor.
#pragma once
#include <cuda_runtime.h>

#include "fft.cuh"
#include "layout.cuh"
#include "step3.cuh"

namespace sb {

// FP32 tiles of the step-2 kernels (measured: 4 z-columns beat 8, 2 x-rows
// beat 1 and 4)
constexpr int MIXED_KB = 4, MIXED_RB = 2;

void mixed_mean_profiles(cudaStream_t s, const float2* stf, double* meanp, const Dims& g);
void mixed_zinv(cudaStream_t s, dim3 grid, size_t smem, const float2* stf, float2* zb, const Dims& g,
                const FFTPlan& plan, const float2* tw, const double* alfa, const double* beta);
void mixed_xpass(cudaStream_t s, dim3 grid, size_t smem, const float2* zb, float2* xb, const Dims& g,
                 const FFTPlan& plan, const float2* tw, const double* dyi, double dxi, double dzi, double rot,
                 unsigned long long* cfl, const double* meanp, Fringe fr);
void mixed_zfwd(cudaStream_t s, dim3 grid, size_t smem, const float2* xb, float2* stf, const Dims& g,
                const FFTPlan& plan, const float2* tw, const double* meanp, double rot);
void mixed_pencil_hom(cudaStream_t s, const PencilBufs& B, const Dims& g, const double* alfa, const double* beta,
                      double re, double anbn, double* vh, double* hs, double* cf);
void mixed_pencil(cudaStream_t s, const PencilBufs& B, const Dims& g, const double* alfa, const double* beta,
                  double re, RKc rk, const double* vh, const double* hs, double* cf);
// one warp per pencil (pencil_warp.cuh); false when ny is outside its range
bool mixed_pencil_warp(cudaStream_t s, const PencilBufs& B, const Dims& g, const double* alfa, const double* beta,
                       double re, RKc rk);
void mixed_mean(cudaStream_t s, const MeanArgs& M, const Dims& g, double re, RKc rk);

}  // namespace sb
