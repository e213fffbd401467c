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
// run here with tcgen05.mma kind::tf32 in the 3xTF32 split: T = T_hi + T_lo
// and IN = X_hi + X_lo rounded to TF32, D = T_hi X_hi + T_hi X_lo + T_lo X_hi
// accumulated in FP32 in tensor memory (the dropped T_lo X_lo is below FP32
// rounding).
//
// Even/odd folding (N = 2H even): cos(pi (N-j) k / N) = (-1)^k cos(pi j k / N),
// so each transform splits into two half-size GEMMs, half the MMA work:
//   forward  a_{2m}   = sum_{j<=H} Fe[m][j] P_j,  P_j = u_j + u_{N-j} (j < H), P_H = u_H
//            a_{2m+1} = sum_{j<H}  Fo[m][j] M_j,  M_j = u_j - u_{N-j}
//   inverse  E_j = sum_{m<=H} Ie[j][m] a_{2m},  O_j = sum_{m<H} Io[j][m] a_{2m+1},
//            u_j = E_j + O_j, u_{N-j} = E_j - O_j (j < H), u_H = E_H,
// with Fe = s w_j cos(2 pi j m / N) / (N cbar_{2m}), Fo = s w_j cos(pi j (2m+1) / N) / N,
// Ie = cos(2 pi j m / N), Io = cos(pi j (2m+1) / N).
//
// One CTA (288 threads: eight producer warps, one MMA warp) owns 128 columns (the data is the A operand, M = 128,
// columns as rows); the matrices are the B operands (N = H+1 and H rounded up
// to 16, at most 112).  K is cut into chunks of 16, taken alternately from
// the even and the odd GEMM (e0 o0 e1 o1 ...), accumulated into TMEM
// columns 0.. (even) and 128.. (odd).  The warps specialise in the main loop:
//   * one thread (warp 8) issues the 3xTF32 MMAs of chunk q as soon as its matrix and
//     data stages are full, commits them to the stages' "empty" mbarriers,
//     and keeps the prepared matrix chunks (canonical K-major TF32 tiles, hi
//     and lo, built on the host) two chunks ahead in a three-stage ring by
//     bulk copies (cp.async.bulk, completing on a "full" mbarrier);
//   * warps 0-7 stage the input: for each pair of chunks the rows j and
//     N-j (forward) or 2m and 2m+1 (inverse) are loaded once, a pair ahead in
//     registers, folded, split into hi/lo TF32 and transposed to K-major in
//     16-byte shared-memory stores into a two-stage ring (even chunk in
//     stage 0, odd in stage 1), then each stage's "full" mbarrier is arrived
//     on (after a proxy fence);
// so the tensor pipe sees chunk after chunk without a CTA-wide barrier in
// the loop.  Every wait is bounded; after the loop one commit covers every
// MMA issued, and every exit waits (bounded) for it and for the copies in
// flight before TMEM is freed.  Epilogue: a warp reads its 32 TMEM lanes
// (data columns); forward, warp group 0 writes the even rows and group 1
// the odd rows; inverse, both groups combine E and O of their share of j
// into rows j and N-j.  A warp's stores of one output row cover 32
// consecutive columns.  75 KB of shared memory and 256 TMEM columns: two
// CTAs per SM, whose epilogues and main loops overlap.
#pragma once
#include "sgs_mlp.cuh"

namespace sb {

constexpr int CHB_TILE = 128;                                 // data columns per CTA (MMA M)
constexpr int CHB_KC = 16;                                    // K rows per chunk
constexpr int CHB_NMAX = 112;                                 // rows of a half matrix (MMA N), >= H + 1
constexpr int CHB_MAX_NY = 2 * (CHB_NMAX - 1) + 1;            // ny = N + 1 with H + 1 <= CHB_NMAX
constexpr int CHB_SBO = (CHB_KC / 4) * 128;                   // bytes between 8-row groups
constexpr int CHB_A_BYTES = CHB_NMAX * CHB_KC * 4;            // one TF32 tile of a half matrix
constexpr int CHB_B_BYTES = CHB_TILE * CHB_KC * 4;            // one TF32 tile of the input
constexpr int CHB_CHUNK_BYTES = 2 * CHB_A_BYTES;              // hi + lo matrix tiles per chunk
constexpr int CHB_MSTAGES = 3;                                // matrix ring
constexpr int CHB_DSTAGE = 2 * CHB_B_BYTES;                   // data hi, lo
constexpr int CHB_DATA0 = CHB_MSTAGES * CHB_CHUNK_BYTES;      // offset of the two data stages
constexpr int CHB_BARS = CHB_DATA0 + 2 * CHB_DSTAGE;          // offset of the mbarriers
constexpr int CHB_SMEM = CHB_BARS + 128;
constexpr int CHB_TMEM_COLS = 256;                            // even accumulator at 0, odd at 128
constexpr int CHB_ODD_COL = 128;
// chunk counts of the folded GEMMs for ny = n (N = n - 1 = 2H)
SB_HD __forceinline__ int chb_even_chunks(int n) { return ((n - 1) / 2 + 1 + CHB_KC - 1) / CHB_KC; }
SB_HD __forceinline__ int chb_odd_chunks(int n) { return ((n - 1) / 2 + CHB_KC - 1) / CHB_KC; }
// chunk q of the interleaved sequence e0 o0 e1 o1 ...: odd part?, index in its part
SB_HD __forceinline__ bool chb_is_odd(int q, int no) { return q < 2 * no && (q & 1); }
SB_HD __forceinline__ int chb_part_index(int q) { return q >> 1; }
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
  const float* in;               // field f, row j, column c at in[f * in_fs + j * ld + c]
  size_t in_fs;
  float* out;
  size_t out_fs;
  int ncol;                      // columns transformed: 2 (p1 - p0), from pencil p0 on
  int ld;                        // row stride (2 NP)
  int p0;                        // first pencil (the columns start at 2 p0 of the full field)
  int n;                         // ny = N + 1, N = 2H
  int inverse;                   // 0: physical -> Chebyshev, 1: Chebyshev -> physical
  int ne, no;                    // K chunks of the even and the odd GEMM
  int nre, nro;                  // MMA N of the even and the odd GEMM (H+1, H rounded up to 16)
  const unsigned char* mat;      // ne + no chunks in the order e0 o0 e1 o1 ..., each (hi, lo) tiles
  int skip_oddball, nx2, zodd;   // inverse of step 3: leave the kz = -nz/2 plane alone
  int* err;
  int wait_limit;                // iterations of each bounded wait of the main loop (<= 0: MLP_WAIT_LIMIT)
  int test_timeout;              // 1: the MMA thread first waits on a barrier nothing completes
};

__device__ __forceinline__ void chb_bulk_load(unsigned dst, const void* src, unsigned bytes, unsigned mbar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// Input of chunk pair i (K rows 16 i .. 16 i + 15 of the folded GEMMs,
// columns c0 .. c0+127): each of the 128 producer threads (pt) loads, for
// CHB_ITEMS groups of four K rows of one column, the two rows each K row
// needs -- u_j and u_{N-j} (forward) or a_{2m} and a_{2m+1} (inverse) -- into
// registers, and later stores the even and the odd tile split into hi/lo
// TF32 (one 16-byte store per group, part and tile).
constexpr int CHB_PRODUCERS = 256;                 // warps 0-7 stage the data
constexpr int CHB_THREADS = CHB_PRODUCERS + 32;     // warp 8: MMA issue and matrix copies
constexpr int CHB_ITEMS = CHB_TILE * (CHB_KC / 4) / CHB_PRODUCERS;

struct ChbPair {
  float x[CHB_ITEMS][4], y[CHB_ITEMS][4];
};

__device__ __forceinline__ void chb_load_pair(const ChebTCArgs& a, const float* __restrict__ in, int c0, int i,
                                              int pt, ChbPair& p) {
  const int N = a.n - 1, H = N / 2;
#pragma unroll
  for (int k = 0; k < CHB_ITEMS; ++k) {
    const int it = pt + CHB_PRODUCERS * k;
    const int r = it % CHB_TILE;
    const int g4 = it / CHB_TILE;
    const int col = c0 + r;
    const bool cv = col < a.ncol;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int m = i * CHB_KC + 4 * g4 + s;  // K index of both GEMMs
      int r0, r1;                              // rows of the two values
      bool v0, v1;
      if (a.inverse) {
        r0 = 2 * m; r1 = 2 * m + 1; v0 = m <= H; v1 = m < H;
      } else {
        r0 = m; r1 = N - m; v0 = m <= H; v1 = m < H;
      }
      p.x[k][s] = (cv && v0) ? in[(size_t)r0 * a.ld + col] : 0.f;
      p.y[k][s] = (cv && v1) ? in[(size_t)r1 * a.ld + col] : 0.f;
    }
  }
}

// odd = 0: the even tile (P or a_even), odd = 1: the odd tile (M or a_odd)
__device__ __forceinline__ void chb_store_tile(const ChebTCArgs& a, const ChbPair& p, int odd, int i, int pt,
                                               unsigned char* Bhi, unsigned char* Blo) {
  const int H = (a.n - 1) / 2;
#pragma unroll
  for (int k = 0; k < CHB_ITEMS; ++k) {
    const int it = pt + CHB_PRODUCERS * k;
    const int r = it % CHB_TILE;
    const int g4 = it / CHB_TILE;
    float v[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int m = i * CHB_KC + 4 * g4 + s;
      if (a.inverse)
        v[s] = odd ? p.y[k][s] : p.x[k][s];
      else if (odd)
        v[s] = p.x[k][s] - p.y[k][s];                      // M_m (zero past H-1)
      else
        v[s] = (m < H) ? p.x[k][s] + p.y[k][s] : p.x[k][s];  // P_m, P_H = u_H
    }
    float4 hi, lo;
    hi.x = to_tf32(v[0]); lo.x = to_tf32(v[0] - hi.x);
    hi.y = to_tf32(v[1]); lo.y = to_tf32(v[1] - hi.y);
    hi.z = to_tf32(v[2]); lo.z = to_tf32(v[2] - hi.z);
    hi.w = to_tf32(v[3]); lo.w = to_tf32(v[3] - hi.w);
    *reinterpret_cast<float4*>(Bhi + chb_canon(r, 4 * g4)) = hi;
    *reinterpret_cast<float4*>(Blo + chb_canon(r, 4 * g4)) = lo;
  }
}

__global__ void __launch_bounds__(CHB_THREADS, 2) k_cheb_tc(ChebTCArgs a) {
  extern __shared__ __align__(1024) unsigned char sm[];
  // matrix stage m (hi | lo) at m * CHB_CHUNK_BYTES; data stage d (hi | lo):
  // d = 0 holds the even chunks, d = 1 the odd ones
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
  const int ne = a.ne, no = a.no, nch = a.ne + a.no;
  // the k-th use of a stage (chunk q = stage + k * stages) completes phase k
  auto mpar = [](int q) { return (unsigned)((q / CHB_MSTAGES) & 1); };
  auto dpar = [](int q) { return (unsigned)((q >> 1) & 1); };
  int issued = 0, consumed = 0;  // MMA thread: matrix copies issued / waited for
  const bool mma_thread = t == CHB_PRODUCERS;
  const int limit = a.wait_limit > 0 ? a.wait_limit : MLP_WAIT_LIMIT;
  if (mma_thread) {
    const unsigned idesc_e = chb_idesc(CHB_TILE, a.nre), idesc_o = chb_idesc(CHB_TILE, a.nro);
    auto issue_matrix = [&](int q) {
      chb_bulk_load(smem_u32(Mhi(q % CHB_MSTAGES)), a.mat + (size_t)q * CHB_CHUNK_BYTES, CHB_CHUNK_BYTES,
                    mfull0 + 8 * (q % CHB_MSTAGES));
      issued = q + 1;
    };
    issue_matrix(0);
    if (nch > 1) issue_matrix(1);
    // test of the timeout path: accb completes only with the commit after
    // the loop, so this wait runs out as a lost completion would
    if (a.test_timeout && !mlp_wait(accb, 0u, limit)) s_fail = 1;
    for (int q = 0; q < nch && !s_fail; ++q) {
      const int ms = q % CHB_MSTAGES, ds = q & 1;
      const bool odd = chb_is_odd(q, no);
      if (!mlp_wait(mfull0 + 8 * ms, mpar(q), limit)) {
        s_fail = 1;
        break;
      }
      consumed = q + 1;
      if (!mlp_wait(dfull0 + 8 * ds, dpar(q), limit)) {
        s_fail = 1;
        break;
      }
      tc_fence_after();
      const unsigned mh = smem_u32(Mhi(ms)), ml = mh + CHB_A_BYTES;
      const unsigned xh = smem_u32(Dhi(ds)), xl = smem_u32(Dlo(ds));
      const unsigned dt = tmem + (odd ? (unsigned)CHB_ODD_COL : 0u);
      const unsigned idesc = odd ? idesc_o : idesc_e;
      const bool first = chb_part_index(q) == 0;
      for (int k = 0; k < CHB_KC / 8; ++k) {
        const unsigned ko = (unsigned)(k * 256);
        const unsigned long long ah = mlp_desc(xh + ko, 128, CHB_SBO), al = mlp_desc(xl + ko, 128, CHB_SBO);
        const unsigned long long bh = mlp_desc(mh + ko, 128, CHB_SBO), bl = mlp_desc(ml + ko, 128, CHB_SBO);
        chb_mma(dt, ah, bh, idesc, (!first || k > 0) ? 1u : 0u);
        chb_mma(dt, ah, bl, idesc, 1u);
        chb_mma(dt, al, bh, idesc, 1u);
      }
      mlp_commit(dempty0 + 8 * ds);
      mlp_commit(mempty0 + 8 * ms);
      if (q + 2 < nch) {
        // matrix stage of chunk q+2 was last read by chunk q-1
        if (q >= 1 && !mlp_wait(mempty0 + 8 * ((q - 1) % CHB_MSTAGES), mpar(q - 1), limit)) {
          s_fail = 1;
          break;
        }
        issue_matrix(q + 2);
      }
    }
    // arrives when every MMA issued above has completed (also after a failure)
    mlp_commit(accb);
  } else if (t < CHB_PRODUCERS) {
    const int pt = t;
    ChbPair pa, pb;
    chb_load_pair(a, in, c0, 0, pt, pa);
    if (ne > 1) chb_load_pair(a, in, c0, 1, pt, pb);
    // pair i: even chunk (chunk 2i, stage 0), then odd chunk (2i+1, stage 1)
    auto stage = [&](int i, ChbPair& p) -> bool {
      for (int odd = 0; odd < 2; ++odd) {
        if (odd && i >= no) break;
        const int q = 2 * i + odd;
        // the stage was last read by chunk q-2
        if (q >= 2 && !mlp_wait(dempty0 + 8 * odd, dpar(q - 2), limit)) return false;
        chb_store_tile(a, p, odd, i, pt, Dhi(odd), Dlo(odd));
        async_proxy_fence();
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(dfull0 + 8 * odd) : "memory");
      }
      if (i + 2 < ne) chb_load_pair(a, in, c0, i + 2, pt, p);
      return true;
    };
    for (int i = 0; i < ne; i += 2) {
      if (!stage(i, pa)) {
        s_fail = 1;
        break;
      }
      if (i + 1 < ne && !stage(i + 1, pb)) {
        s_fail = 1;
        break;
      }
    }
  }
  __syncthreads();
  // the accumulators (every MMA complete), then the copies still in flight
  // (only after a failed wait)
  bool acc_ok = mlp_wait(accb, 0u, MLP_WAIT_LIMIT);
  if (mma_thread)
    for (int q = consumed; q < issued; ++q)
      if (!mlp_wait(mfull0 + 8 * (q % CHB_MSTAGES), mpar(q), MLP_WAIT_LIMIT)) acc_ok = false;
  if (!acc_ok) s_fail = 1;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (!s_fail && warp < 8) {
    // warp w reads TMEM lanes 32 (w % 4) .. +31 (data columns)
    const int N = a.n - 1, H = N / 2;
    const int grp = warp >> 2;
    const int col = c0 + (warp & 3) * 32 + (t & 31);
    const bool keep = col < a.ncol && !(a.skip_oddball && (a.p0 + (col >> 1)) / a.nx2 == a.zodd);
    const unsigned taddr = tmem + ((unsigned)((warp & 3) * 32) << 16);
    if (!a.inverse) {
      // group 0: even rows k = 2m from TMEM columns m; group 1: odd rows
      // k = 2m+1 from columns 128 + m
      const int nm = grp == 0 ? H + 1 : H;
      const unsigned base = taddr + (grp == 0 ? 0u : (unsigned)CHB_ODD_COL);
      for (int kc = 0; 16 * kc < nm; ++kc) {
        float v[16];
        mlp_ld16(base + 16 * kc, v);
        mlp_ld_wait();
        if (keep) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int m = 16 * kc + i;
            if (m < nm) out[(size_t)(2 * m + grp) * a.ld + col] = v[i];
          }
        }
      }
    } else {
      // E_j (columns j) and O_j (columns 128 + j): rows j and N - j; the two
      // groups split the j blocks
      const int nkc = (H + 1 + 15) / 16;
      const int k0 = grp == 0 ? 0 : (nkc + 1) / 2, k1 = grp == 0 ? (nkc + 1) / 2 : nkc;
      for (int kc = k0; kc < k1; ++kc) {
        float e[16], o[16];
        mlp_ld16(taddr + 16 * kc, e);
        const bool has_o = 16 * kc < H;  // odd accumulator holds j < H only
        if (has_o) mlp_ld16(taddr + CHB_ODD_COL + 16 * kc, o);
        mlp_ld_wait();
        if (keep) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int j = 16 * kc + i;
            if (j < H) {
              const float ov = has_o ? o[i] : 0.f;
              out[(size_t)j * a.ld + col] = e[i] + ov;
              out[(size_t)(N - j) * a.ld + col] = e[i] - ov;
            } else if (j == H) {
              out[(size_t)j * a.ld + col] = e[i];
            }
          }
        }
      }
    }
  } else if (s_fail && t == 0) {
    atomicExch(a.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(CHB_TMEM_COLS) : "memory");
  }
}

// Host: the two half matrices as (ne + no) chunks, interleaved e0 o0 e1 o1
// ..., each hi and lo TF32 tiles (rows = MMA N index, K-major).  inverse = 0:
// forward (Fe, Fo) with scale s; inverse = 1: synthesis (Ie, Io).
inline float chb_host_tf32(double v) {
  // round to nearest (ties away) to 10 explicit mantissa bits, as cvt.rna.tf32
  float f = (float)v;
  unsigned u;
  memcpy(&u, &f, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  memcpy(&f, &u, 4);
  return f;
}

// element (r, c) of the even (odd = 0) or odd half matrix; 0 outside it
inline long double chb_half_entry(int n, int inverse, int odd, int r, int c, double scale) {
  const int N = n - 1, H = N / 2;
  const long double pi = 3.14159265358979323846264338327950288L;
  if (odd ? (r >= H || c >= H) : (r > H || c > H)) return 0.0L;
  if (inverse) {
    // Ie[j][m] = cos(2 pi j m / N), Io[j][m] = cos(pi j (2m+1) / N)
    const long long t = odd ? (long long)r * (2 * c + 1) : 2LL * r * c;
    return cosl(pi * (long double)(t % (2 * N)) / (long double)N);
  }
  // Fe[m][j] = s w_j cos(2 pi j m / N) / (N cbar_{2m}), Fo[m][j] = s w_j cos(pi j (2m+1) / N) / N
  const long long t = odd ? (long long)c * (2 * r + 1) : 2LL * c * r;
  const long double w = (c == 0) ? 1.0L : 2.0L;
  const long double cb = (!odd && (r == 0 || 2 * r == N)) ? 2.0L : 1.0L;
  return (long double)scale * w * cosl(pi * (long double)(t % (2 * N)) / (long double)N) / ((long double)N * cb);
}

inline void chb_build_matrix(int n, int inverse, double scale, std::vector<unsigned char>& img) {
  const int ne = chb_even_chunks(n), no = chb_odd_chunks(n);
  img.assign((size_t)(ne + no) * CHB_CHUNK_BYTES, 0);
  for (int q = 0; q < ne + no; ++q) {
    const int odd = chb_is_odd(q, no) ? 1 : 0, pi = chb_part_index(q);
    unsigned char* base = img.data() + (size_t)q * CHB_CHUNK_BYTES;
    for (int r = 0; r < CHB_NMAX; ++r)
      for (int kk = 0; kk < CHB_KC; ++kk) {
        const long double v = chb_half_entry(n, inverse, odd, r, pi * CHB_KC + kk, scale);
        const float hi = chb_host_tf32((double)v);
        const float lo = chb_host_tf32((double)(v - (long double)hi));
        memcpy(base + chb_canon(r, kk), &hi, 4);
        memcpy(base + CHB_A_BYTES + chb_canon(r, kk), &lo, 4);
      }
  }
}

}  // namespace sb
