// Chebyshev transforms of the mixed-precision path on the tensor cores.
//
// Along y the physical <-> Chebyshev transform of every pencil is one dense
// (N+1) x (N+1) matrix (N = ny - 1), the same for all pencils:
//   forward  a_k = s / (N cbar_k) sum_j w_j u_j cos(pi j k / N)
//            (w_j = 1 at j = 0, N, else 2; cbar = 2 at k = 0, N, else 1;
//             s the caller's scale)
//   inverse  u_j = sum_k a_k cos(pi j k / N)
// -- the DCT-I that the FP64 path computes by FFT (step3.cuh k_cheb, the
// conventions of bla/cvecfft_acc.f vchbf/vchbb with linearbl.f's scaling).
// With the pencils' real and imaginary parts as 2 NP columns it is a GEMM,
// OUT (n x 2NP) = T (n x n) * IN (n x 2NP), run here with tcgen05.mma
// kind::tf32 in the 3xTF32 split: T = T_hi + T_lo and IN = X_hi + X_lo rounded
// to TF32, D = T_hi X_hi + T_hi X_lo + T_lo X_hi accumulated in FP32 in tensor
// memory (the dropped T_lo X_lo is below FP32 rounding).
//
// One CTA (256 threads) owns 128 columns (the data is the A operand, M = 128,
// columns as rows), the matrix is the B operand (N = 208 >= n output rows,
// rows >= n zero), K = y in chunks of 16 (two MMA steps of 8).  The warps
// specialise during the main loop:
//   * thread 0 issues the 3xTF32 MMAs of chunk q as soon as its matrix and
//     data stages are full, commits them to the stages' "empty" mbarriers,
//     and keeps the prepared matrix chunks (canonical K-major TF32 tiles, hi
//     and lo, built on the host) two chunks ahead in a three-stage ring by
//     bulk copies (cp.async.bulk, completing on a "full" mbarrier);
//   * warps 4-7 stage the input: global loads two chunks ahead in
//     registers, the split into hi/lo TF32 and the transpose to K-major in
//     16-byte shared-memory stores into a two-stage ring, then arrive on the
//     stage's "full" mbarrier (after a proxy fence);
// so the tensor pipe sees chunk after chunk without a CTA-wide barrier in
// the loop.  Every wait is bounded; after the loop one commit covers every
// MMA issued, and every exit waits (bounded) for it and for the copies in
// flight before TMEM is freed.  Accumulator: 208 TMEM columns (lane = data
// column, TMEM column = output row); in the epilogue the two warp groups
// split the output rows, a warp's stores of one output row cover 32
// consecutive columns.  110 KB of shared memory and 256 TMEM columns: two
// CTAs per SM, whose epilogues and main loops overlap.
#pragma once
#include "sgs_mlp.cuh"

namespace sb {

constexpr int CHB_TILE = 128;                                 // data columns per CTA (MMA M)
constexpr int CHB_KC = 16;                                    // K rows per chunk
constexpr int CHB_MROWS = 208;                                // matrix rows (MMA N), >= ny
constexpr int CHB_SBO = (CHB_KC / 4) * 128;                   // bytes between 8-row groups
constexpr int CHB_A_BYTES = CHB_MROWS * CHB_KC * 4;           // one TF32 tile of the matrix
constexpr int CHB_B_BYTES = CHB_TILE * CHB_KC * 4;            // one TF32 tile of the input
constexpr int CHB_CHUNK_BYTES = 2 * CHB_A_BYTES;              // hi + lo matrix tiles per chunk
constexpr int CHB_MSTAGES = 3;                                // matrix ring
constexpr int CHB_DSTAGE = 2 * CHB_B_BYTES;                   // data hi, lo
constexpr int CHB_DATA0 = CHB_MSTAGES * CHB_CHUNK_BYTES;      // offset of the two data stages
constexpr int CHB_BARS = CHB_DATA0 + 2 * CHB_DSTAGE;          // offset of the mbarriers
constexpr int CHB_SMEM = CHB_BARS + 128;
constexpr int CHB_TMEM_COLS = 256;                            // 208 used
// byte offset of (row r, k) in a canonical K-major TF32 tile with CHB_KC columns
SB_HD __forceinline__ int chb_canon(int r, int k) { return (r >> 3) * CHB_SBO + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4; }

// instruction descriptor: FP32 accumulator, TF32 A and B, both K-major
__host__ __device__ constexpr unsigned chb_idesc(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(n >> 3) << 17) | ((unsigned)(m >> 4) << 24);
}

__device__ __forceinline__ void chb_mma(unsigned dtmem, unsigned long long ad, unsigned long long bd, unsigned idesc,
                                        unsigned acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ float to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

struct ChebTCArgs {
  const float* in;               // field f, row j, column c at in[f * in_fs + j * ncol + c]
  size_t in_fs;
  float* out;
  size_t out_fs;
  int ncol;                      // 2 NP
  int n;                         // ny
  int nchunks;                   // ceil(n / CHB_KC)
  const unsigned char* mat;      // nchunks x (hi, lo) canonical tiles of the matrix
  int skip_oddball, nx2, zodd;   // inverse of step 3: leave the kz = -nz/2 plane alone
  int* err;
};

__device__ __forceinline__ void chb_bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned mbar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// Input chunk q (rows q*KC .. +KC of columns c0 .. c0+127): each of the 128
// producer threads (pt) loads CHB_ITEMS groups of four rows of one column
// into registers, and later stores them split into hi/lo TF32 (one 16-byte
// store per group and part).
constexpr int CHB_PRODUCERS = 128;
constexpr int CHB_ITEMS = CHB_TILE * (CHB_KC / 4) / CHB_PRODUCERS;

__device__ __forceinline__ void chb_load_input(const ChebTCArgs& a, const float* __restrict__ in, int c0, int q,
                                               int pt, float (&x)[CHB_ITEMS][4]) {
#pragma unroll
  for (int k = 0; k < CHB_ITEMS; ++k) {
    const int it = pt + CHB_PRODUCERS * k;
    const int r = it % CHB_TILE;
    const int g4 = it / CHB_TILE;
    const int col = c0 + r;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = q * CHB_KC + 4 * g4 + i;
      x[k][i] = (row < a.n && col < a.ncol) ? in[(size_t)row * a.ncol + col] : 0.f;
    }
  }
}

__device__ __forceinline__ void chb_store_input(const float (&x)[CHB_ITEMS][4], int pt, unsigned char* Bhi,
                                                unsigned char* Blo) {
#pragma unroll
  for (int k = 0; k < CHB_ITEMS; ++k) {
    const int it = pt + CHB_PRODUCERS * k;
    const int r = it % CHB_TILE;
    const int g4 = it / CHB_TILE;
    float4 hi, lo;
    hi.x = to_tf32(x[k][0]); lo.x = to_tf32(x[k][0] - hi.x);
    hi.y = to_tf32(x[k][1]); lo.y = to_tf32(x[k][1] - hi.y);
    hi.z = to_tf32(x[k][2]); lo.z = to_tf32(x[k][2] - hi.z);
    hi.w = to_tf32(x[k][3]); lo.w = to_tf32(x[k][3] - hi.w);
    *reinterpret_cast<float4*>(Bhi + chb_canon(r, 4 * g4)) = hi;
    *reinterpret_cast<float4*>(Blo + chb_canon(r, 4 * g4)) = lo;
  }
}

__global__ void __launch_bounds__(256, 2) k_cheb_tc(ChebTCArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  // matrix stage m (hi | lo) at m * CHB_CHUNK_BYTES; data stage d (hi | lo)
  auto Mhi = [&](int m) { return sm + m * CHB_CHUNK_BYTES; };
  auto Dhi = [&](int d) { return sm + CHB_DATA0 + d * CHB_DSTAGE; };
  auto Dlo = [&](int d) { return sm + CHB_DATA0 + d * CHB_DSTAGE + CHB_B_BYTES; };
  // mbarriers: mfull[3], mempty[3], dfull[2], dempty[2], acc
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(sm + CHB_BARS);
  unsigned* tslot = reinterpret_cast<unsigned*>(sm + CHB_BARS + 96);
  __shared__ int s_fail;
  const int t = threadIdx.x, warp = t >> 5;
  const int f = blockIdx.y;
  const int c0 = blockIdx.x * CHB_TILE;
  const float* __restrict__ in = a.in + (size_t)f * a.in_fs;
  float* __restrict__ out = a.out + (size_t)f * a.out_fs;
  const unsigned mfull0 = smem_u32(&bars[0]), mempty0 = smem_u32(&bars[3]);
  const unsigned dfull0 = smem_u32(&bars[6]), dempty0 = smem_u32(&bars[8]), accb = smem_u32(&bars[10]);
  if (t == 0) {
    s_fail = 0;
    for (int i = 0; i < 11; ++i) {
      const unsigned cnt = (i == 6 || i == 7) ? (unsigned)CHB_PRODUCERS : 1u;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&bars[i])), "r"(cnt) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(CHB_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = *tslot;
  const int nch = a.nchunks;
  // the k-th use of a stage (chunk q = stage + k * stages) completes phase k
  auto mpar = [](int q) { return (unsigned)((q / CHB_MSTAGES) & 1); };
  auto dpar = [](int q) { return (unsigned)((q >> 1) & 1); };
  int issued = 0, consumed = 0;  // thread 0: matrix copies issued / waited for
  if (t == 0) {
    constexpr unsigned IDESC = chb_idesc(CHB_TILE, CHB_MROWS);
    auto issue_matrix = [&](int q) {
      chb_bulk_load(smem_u32(Mhi(q % CHB_MSTAGES)), a.mat + (size_t)q * CHB_CHUNK_BYTES, CHB_CHUNK_BYTES,
                    mfull0 + 8 * (q % CHB_MSTAGES));
      issued = q + 1;
    };
    issue_matrix(0);
    if (nch > 1) issue_matrix(1);
    for (int q = 0; q < nch; ++q) {
      const int ms = q % CHB_MSTAGES, ds = q & 1;
      if (!mlp_wait(mfull0 + 8 * ms, mpar(q), MLP_WAIT_LIMIT)) {
        s_fail = 1;
        break;
      }
      consumed = q + 1;
      if (!mlp_wait(dfull0 + 8 * ds, dpar(q), MLP_WAIT_LIMIT)) {
        s_fail = 1;
        break;
      }
      tc_fence_after();
      const unsigned mh = smem_u32(Mhi(ms)), ml = mh + CHB_A_BYTES;
      const unsigned xh = smem_u32(Dhi(ds)), xl = smem_u32(Dlo(ds));
      for (int k = 0; k < CHB_KC / 8; ++k) {
        const unsigned ko = (unsigned)(k * 256);
        const unsigned long long ah = mlp_desc(xh + ko, 128, CHB_SBO), al = mlp_desc(xl + ko, 128, CHB_SBO);
        const unsigned long long bh = mlp_desc(mh + ko, 128, CHB_SBO), bl = mlp_desc(ml + ko, 128, CHB_SBO);
        chb_mma(tmem, ah, bh, IDESC, (q > 0 || k > 0) ? 1u : 0u);
        chb_mma(tmem, ah, bl, IDESC, 1u);
        chb_mma(tmem, al, bh, IDESC, 1u);
      }
      mlp_commit(dempty0 + 8 * ds);
      mlp_commit(mempty0 + 8 * ms);
      if (q + 2 < nch) {
        // matrix stage of chunk q+2 was last read by chunk q-1
        if (q >= 1 && !mlp_wait(mempty0 + 8 * ((q - 1) % CHB_MSTAGES), mpar(q - 1), MLP_WAIT_LIMIT)) {
          s_fail = 1;
          break;
        }
        issue_matrix(q + 2);
      }
    }
    // arrives when every MMA issued above has completed (also after a failure)
    mlp_commit(accb);
  } else if (warp >= 4) {
    const int pt = t - 128;
    float x0[CHB_ITEMS][4], x1[CHB_ITEMS][4];
    chb_load_input(a, in, c0, 0, pt, x0);
    if (nch > 1) chb_load_input(a, in, c0, 1, pt, x1);
    auto stage = [&](int q, float (&x)[CHB_ITEMS][4]) -> bool {
      const int ds = q & 1;
      // data stage of chunk q was last read by chunk q-2
      if (q >= 2 && !mlp_wait(dempty0 + 8 * ds, dpar(q - 2), MLP_WAIT_LIMIT)) return false;
      chb_store_input(x, pt, Dhi(ds), Dlo(ds));
      async_proxy_fence();
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(dfull0 + 8 * ds) : "memory");
      if (q + 2 < nch) chb_load_input(a, in, c0, q + 2, pt, x);
      return true;
    };
    for (int q = 0; q < nch; q += 2) {
      if (!stage(q, x0)) {
        s_fail = 1;
        break;
      }
      if (q + 1 < nch && !stage(q + 1, x1)) {
        s_fail = 1;
        break;
      }
    }
  }
  __syncthreads();
  // the accumulator (every MMA complete), then the copies still in flight
  // (only after a failed wait)
  bool acc_ok = mlp_wait(accb, 0u, MLP_WAIT_LIMIT);
  if (t == 0)
    for (int q = consumed; q < issued; ++q)
      if (!mlp_wait(mfull0 + 8 * (q % CHB_MSTAGES), mpar(q), MLP_WAIT_LIMIT)) acc_ok = false;
  if (!acc_ok) s_fail = 1;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (!s_fail) {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (data columns);
    // TMEM column k is output row k; the two warp groups split the rows
    constexpr int KG = CHB_MROWS / 16;
    const int grp = warp >> 2;
    const int kc0 = grp == 0 ? 0 : (KG + 1) / 2, kc1 = grp == 0 ? (KG + 1) / 2 : KG;
    const int col = c0 + (warp & 3) * 32 + (t & 31);
    const bool keep = col < a.ncol && !(a.skip_oddball && (col >> 1) / a.nx2 == a.zodd);
    const unsigned taddr = tmem + ((unsigned)((warp & 3) * 32) << 16);
    for (int kc = kc0; kc < kc1; ++kc) {
      float v[16];
      mlp_ld16(taddr + 16 * kc, v);
      mlp_ld_wait();
      if (keep) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int row = 16 * kc + i;
          if (row < a.n) out[(size_t)row * a.ncol + col] = v[i];
        }
      }
    }
  } else if (t == 0) {
    atomicExch(a.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CHB_TMEM_COLS) : "memory");
  }
}

// Host: the transform matrix as nchunks x (hi, lo) TF32 tiles.  inverse = 0:
// forward with scale s; inverse = 1: synthesis.
inline float chb_host_tf32(double v) {
  // round to nearest (ties away) to 10 explicit mantissa bits, as cvt.rna.tf32
  float f = (float)v;
  unsigned u;
  memcpy(&u, &f, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  memcpy(&f, &u, 4);
  return f;
}

inline void chb_build_matrix(int n, int inverse, double scale, std::vector<unsigned char>& img) {
  const int N = n - 1;
  const int nch = (n + CHB_KC - 1) / CHB_KC;
  img.assign((size_t)nch * CHB_CHUNK_BYTES, 0);
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) {
      long double v;
      if (inverse) {
        v = cosl(pi * (long double)((long long)r * c % (2 * N)) / (long double)N);
      } else {
        const long double w = (c == 0 || c == N) ? 1.0L : 2.0L;
        const long double cb = (r == 0 || r == N) ? 2.0L : 1.0L;
        v = (long double)scale * w * cosl(pi * (long double)((long long)r * c % (2 * N)) / (long double)N) /
            ((long double)N * cb);
      }
      const float hi = chb_host_tf32((double)v);
      const float lo = chb_host_tf32((double)(v - (long double)hi));
      const int q = c / CHB_KC, kk = c % CHB_KC;
      unsigned char* base = img.data() + (size_t)q * CHB_CHUNK_BYTES;
      memcpy(base + chb_canon(r, kk), &hi, 4);
      memcpy(base + CHB_A_BYTES + chb_canon(r, kk), &lo, 4);
    }
}

}  // namespace sb
