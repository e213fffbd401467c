// Learned SGS model: a small MLP maps the resolved velocity gradient and the
// wall distance to the SGS stress, on the 5th-generation tensor cores.
// No counterpart in the reference; it fills the slot of the eddy-viscosity
// stress (bla/les.f:1620-1640, taur/taui), and the stress then goes through
// the same divergence (bla/sgs_stress.f) and step-2 forcing as iles = 2.
//
//   features x (10):  x_3i+j = s_in * du_i/dx_j (i, j = x, y, z),
//                     x_9    = s_y * (1 - |y|)   (wall distance)
//   h1 = tanh(W1 x + b1)  (64)   h2 = tanh(W2 h1 + b2)  (64)
//   tau_ij = s_out * (W3 h2 + b3)   (6: 11 12 13 22 23 33)
//
// Arithmetic: weights, x, h1, h2 rounded to BF16 (round to nearest even),
// products accumulated in FP32 in tensor memory, biases in FP32, tanh by the
// hardware approximation (tanh.approx.f32, relative error ~2^-11, below the
// BF16 rounding of the activations that follows it).
//
// One CTA of 128 threads takes 128 points at a time (thread t = row t):
// each layer is tcgen05.mma kind::f16 with M = 128 (K = 16 steps; N = 64, 64,
// 16), A and B in shared memory in the canonical K-major layout without
// swizzle (8-row x 16-byte core matrices: K-adjacent cores 128 bytes apart
// (LBO), 8-row groups K/8 * 128 bytes apart (SBO)), the FP32 accumulator in
// 128 TMEM columns; tcgen05.ld brings each thread its row back for the bias,
// tanh and BF16 rounding that form the next layer's A operand.  One elected
// thread issues the MMAs and commits them to an mbarrier; every wait on it is
// bounded, and a wait that runs out sets the error word, lets the MMA finish
// (again bounded), frees the TMEM and returns.
#pragma once
#include <cuda_bf16.h>

#include "fft.cuh"

namespace sb {

constexpr int MLP_IN = 10, MLP_H = 64, MLP_OUT = 6, MLP_N3 = 16, MLP_ROWS = 128;
constexpr int MLP_TMEM_COLS = 128;

// Shared-memory image of the weights (canonical K-major BF16 tiles) and
// biases, built on the host and copied into every CTA.
constexpr int MLP_B1_BYTES = MLP_H * 16 * 2;      // 64 x 16 (K 10 -> 16)
constexpr int MLP_B2_BYTES = MLP_H * MLP_H * 2;   // 64 x 64
constexpr int MLP_B3_BYTES = MLP_N3 * MLP_H * 2;  // 16 x 64 (rows 6..15 zero)
constexpr int MLP_BIAS_FLOATS = MLP_H + MLP_H + MLP_N3;
constexpr int MLP_IMAGE_BYTES = MLP_B1_BYTES + MLP_B2_BYTES + MLP_B3_BYTES + MLP_BIAS_FLOATS * 4;

// byte offset of element (r, k) in a canonical K-major tile of kcols columns
SB_HD __forceinline__ int mlp_canon(int r, int k, int kcols) {
  return (r >> 3) * (kcols / 8) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

struct MlpArgs {
  const unsigned char* image;  // MLP_IMAGE_BYTES, 16-byte aligned
  int mode;                    // 0: x[n][10] -> y[n][6]; 1: phys gradients -> tau fields
  long long n;                 // points
  const float* x;              // mode 0
  float* y;                    // mode 0
  const double* grad;          // mode 1: [9][n] physical du_i/dx_j
  double* tau;                 // mode 1: [6][n]
  int plane;                   // mode 1: points per y-plane (nz * nx)
  int nyp;
  float s_in, s_y, s_out;
  int* err;                    // set to 1 if a wait ran out
  int wait_limit;              // iterations of each bounded wait of the main loop (<= 0: MLP_WAIT_LIMIT)
  int test_timeout;            // 1: first wait on a barrier nothing completes (tests the timeout path)
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// sm100 shared-memory matrix descriptor: start, LBO, SBO (all >> 4),
// version 1, base offset 0, no swizzle
__device__ __forceinline__ unsigned long long mlp_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((addr & 0x3FFFFu) >> 4) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major
__host__ __device__ constexpr unsigned mlp_idesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(m >> 4) << 24);
}

__device__ __forceinline__ void mlp_mma(unsigned dtmem, unsigned long long ad, unsigned long long bd, unsigned idesc,
                                        unsigned acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mlp_commit(unsigned mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool mlp_wait(unsigned mbar, unsigned phase, int limit) {
  for (int i = 0; i < limit; ++i) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void mlp_ld16(unsigned taddr, float* v) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void mlp_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ unsigned pack_bf16x2(float a, float b) {
  const __nv_bfloat16 x = __float2bfloat16_rn(a), y = __float2bfloat16_rn(b);
  return (unsigned)__bfloat16_as_ushort(x) | ((unsigned)__bfloat16_as_ushort(y) << 16);
}

// 8 values -> one 16-byte row segment of a core matrix
__device__ __forceinline__ void mlp_store8(unsigned char* tile, int r, int kc, int kcols, const float* v) {
  uint4 q;
  q.x = pack_bf16x2(v[0], v[1]);
  q.y = pack_bf16x2(v[2], v[3]);
  q.z = pack_bf16x2(v[4], v[5]);
  q.w = pack_bf16x2(v[6], v[7]);
  *reinterpret_cast<uint4*>(tile + mlp_canon(r, kc * 8, kcols)) = q;
}

// Dynamic shared memory layout (bytes): A1 4096 | A 16384 | B1 | B2 | B3 |
// biases | mbarrier 8 | TMEM address 4.  The launch asks for more than it uses
// so that at most four CTAs (4 x 128 TMEM columns) share an SM.
constexpr int MLP_SMEM_A1 = 0;
constexpr int MLP_SMEM_A = 4096;
constexpr int MLP_SMEM_W = MLP_SMEM_A + MLP_ROWS * MLP_H * 2;
constexpr int MLP_SMEM_BAR = MLP_SMEM_W + ((MLP_IMAGE_BYTES + 15) / 16) * 16;
constexpr int MLP_SMEM_USED = MLP_SMEM_BAR + 16;
constexpr int MLP_SMEM_LAUNCH = 56 * 1024;
constexpr int MLP_WAIT_LIMIT = 1 << 20;

__device__ __forceinline__ float mlp_tanh(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// planes whose wall-distance feature is tabulated per CTA (larger grids
// compute it per point)
constexpr int MLP_YTAB = 512;

__global__ void __launch_bounds__(128) k_sgs_mlp(MlpArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* A1 = sm + MLP_SMEM_A1;
  unsigned char* A = sm + MLP_SMEM_A;
  unsigned char* W = sm + MLP_SMEM_W;
  unsigned char* B1 = W;
  unsigned char* B2 = W + MLP_B1_BYTES;
  unsigned char* B3 = B2 + MLP_B2_BYTES;
  const float* bias = reinterpret_cast<const float*>(B3 + MLP_B3_BYTES);
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm + MLP_SMEM_BAR);
  unsigned* tslot = reinterpret_cast<unsigned*>(sm + MLP_SMEM_BAR + 8);
  __shared__ int s_fail;
  __shared__ float s_ywall[MLP_YTAB];  // x_9 = s_y (1 - |y|) of each plane
  const int t = threadIdx.x, warp = t >> 5;
  const bool ytab = a.mode == 1 && a.nyp <= MLP_YTAB;
  if (ytab)
    for (int y = t; y < a.nyp; y += blockDim.x) {
      const double eta = cos(3.1415926535897932385 * (double)y / (double)(a.nyp - 1));
      s_ywall[y] = a.s_y * (float)(1.0 - fabs(eta));
    }

  // weights and biases into shared memory
  for (int i = t; i < MLP_IMAGE_BYTES / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(W)[i] = reinterpret_cast<const uint4*>(a.image)[i];
  if (t == 0) {
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(MLP_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tslot;
  const unsigned mb = smem_u32(bar);
  const unsigned lane_base = (unsigned)(warp * 32) << 16;
  unsigned phase = 0;
  bool fail = false;

  const int limit = a.wait_limit > 0 ? a.wait_limit : MLP_WAIT_LIMIT;
  bool mma_pending = false;  // an MMA committed whose completion nobody has seen
  if (a.test_timeout) {
    // the barrier's phase 0 completes only with a commit, and none is made
    // before this wait: it runs out, as a lost completion would
    if (!mlp_wait(mb, phase, limit)) s_fail = 1;
    __syncthreads();
    fail = s_fail != 0;
  }
  const long long ntiles = (a.n + MLP_ROWS - 1) / MLP_ROWS;
  for (long long tile = blockIdx.x; tile < ntiles && !fail; tile += gridDim.x) {
    const long long i = tile * MLP_ROWS + t;
    const bool live = i < a.n;
    // ---- features -> A1 (128 x 16)
    float x[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = 0.f;
    if (live) {
      if (a.mode == 0) {
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) x[k] = a.x[i * MLP_IN + k];
      } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) x[k] = a.s_in * (float)a.grad[(long long)k * a.n + i];
        const int y = (int)(i / a.plane);
        if (ytab) {
          x[9] = s_ywall[y];
        } else {
          const double eta = cos(3.1415926535897932385 * (double)y / (double)(a.nyp - 1));
          x[9] = a.s_y * (float)(1.0 - fabs(eta));
        }
      }
    }
    mlp_store8(A1, t, 0, 16, x);
    mlp_store8(A1, t, 1, 16, x + 8);
    async_proxy_fence();
    tc_fence_before();
    __syncthreads();
    // ---- layer 1: D[0:64) = A1 (128x16) * B1^T
    if (t == 0) {
      tc_fence_after();
      mlp_mma(tmem, mlp_desc(smem_u32(A1), 128, 256), mlp_desc(smem_u32(B1), 128, 256), mlp_idesc(128, 64), 0u);
      mlp_commit(mb);
    }
    mma_pending = true;
    for (int layer = 0; layer < 3; ++layer) {
      const bool ok = mlp_wait(mb, phase, limit);
      if (!ok) s_fail = 1;
      if (ok) mma_pending = false;
      phase ^= 1u;
      tc_fence_after();
      __syncthreads();
      if (s_fail) {
        fail = true;
        break;
      }
      const unsigned dcol = (layer == 1) ? 64u : 0u;
      if (layer < 2) {
        // bias + tanh, BF16 into A (128 x 64)
        const float* b = bias + layer * MLP_H;
        for (int c = 0; c < 4; ++c) {
          float v[16];
          mlp_ld16(tmem + lane_base + dcol + 16 * c, v);
          mlp_ld_wait();
#pragma unroll
          for (int q = 0; q < 16; ++q) v[q] = mlp_tanh(v[q] + b[16 * c + q]);
          mlp_store8(A, t, 2 * c, MLP_H, v);
          mlp_store8(A, t, 2 * c + 1, MLP_H, v + 8);
        }
        async_proxy_fence();
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
          tc_fence_after();
          unsigned char* Bn = (layer == 0) ? B2 : B3;
          const unsigned dn = (layer == 0) ? 64u : 0u;
          const unsigned idn = (layer == 0) ? mlp_idesc(128, 64) : mlp_idesc(128, MLP_N3);
          for (int kc = 0; kc < 4; ++kc)
            mlp_mma(tmem + dn, mlp_desc(smem_u32(A) + 256 * kc, 128, 1024), mlp_desc(smem_u32(Bn) + 256 * kc, 128, 1024),
                    idn, kc > 0 ? 1u : 0u);
          mlp_commit(mb);
        }
        mma_pending = true;
      } else {
        // output layer: columns 0..5 of D
        float v[16];
        mlp_ld16(tmem + lane_base, v);
        mlp_ld_wait();
        if (live) {
          const float* b3 = bias + 2 * MLP_H;
          if (a.mode == 0) {
#pragma unroll
            for (int q = 0; q < MLP_OUT; ++q) a.y[i * MLP_OUT + q] = a.s_out * (v[q] + b3[q]);
          } else {
#pragma unroll
            for (int q = 0; q < MLP_OUT; ++q) a.tau[(long long)q * a.n + i] = (double)(a.s_out * (v[q] + b3[q]));
          }
        }
        tc_fence_before();
        __syncthreads();
      }
    }
  }
  if (fail) {
    if (t == 0) atomicExch(a.err, 1);
    // let the committed MMA whose wait ran out finish before its accumulator
    // columns are freed (the full limit, whatever the main loop's)
    if (mma_pending) mlp_wait(mb, phase ^ 1u, MLP_WAIT_LIMIT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(MLP_TMEM_COLS) : "memory");
  }
}

// Host: BF16 (round to nearest even) weight image in the canonical layout.
inline unsigned short mlp_host_bf16(float f) {
  unsigned u;
  memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (unsigned short)(u >> 16);
}

inline void mlp_build_image(const float* w1, const float* b1, const float* w2, const float* b2, const float* w3,
                            const float* b3, unsigned char* img) {
  memset(img, 0, MLP_IMAGE_BYTES);
  unsigned char* B1 = img;
  unsigned char* B2 = img + MLP_B1_BYTES;
  unsigned char* B3 = B2 + MLP_B2_BYTES;
  auto put = [](unsigned char* tile, int r, int k, int kcols, float v) {
    const unsigned short h = mlp_host_bf16(v);
    memcpy(tile + mlp_canon(r, k, kcols), &h, 2);
  };
  for (int n = 0; n < MLP_H; ++n)
    for (int k = 0; k < MLP_IN; ++k) put(B1, n, k, 16, w1[n * MLP_IN + k]);
  for (int n = 0; n < MLP_H; ++n)
    for (int k = 0; k < MLP_H; ++k) put(B2, n, k, MLP_H, w2[n * MLP_H + k]);
  for (int n = 0; n < MLP_OUT; ++n)
    for (int k = 0; k < MLP_H; ++k) put(B3, n, k, MLP_H, w3[n * MLP_H + k]);
  float* bias = reinterpret_cast<float*>(B3 + MLP_B3_BYTES);
  for (int j = 0; j < MLP_H; ++j) bias[j] = b1[j];
  for (int j = 0; j < MLP_H; ++j) bias[MLP_H + j] = b2[j];
  for (int j = 0; j < MLP_OUT; ++j) bias[2 * MLP_H + j] = b3[j];
}

}  // namespace sb
