// Host side of the C ABI declared in include/simson_b200.h: the resident
// device state, the transform plans and tables, and the launch sequence of one
// RK3/CN substep.  The RK bookkeeping mirrors the reference driver
// (bla/bla.f:1464-1478 first stage, 2382-2397 weights, 2598-2607 time).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/simson_b200.h"
#include "fft.cuh"
#include "layout.cuh"
#include "step2.cuh"
#include "step3.cuh"
#include "stats.cuh"
#include "les.cuh"
#include "les_filter.h"
#include "les_dyn.cuh"
#include "sgs_mlp.cuh"
#include "xys.cuh"
#include "press.cuh"
#include "mlp_train.cuh"

#include <nvtx3/nvToolsExt.h>
#include "mixed.h"
#include "step2_launch.cuh"
#include "cheb_tc.cuh"
#include "pencil_warp.cuh"

using namespace sb;

namespace {

// RK stage weights a_k, b_k, c_k of the 3-stage (Wray) and the 4-stage
// scheme, the values of bla/rkcoeff.f:8-48 (row nst - 3)
const double ANRK[2][4] = {{8. / 15., 5. / 12., 3. / 4., 0.}, {8. / 17., 17. / 60., 5. / 12., 3. / 4.}};
const double BNRK[2][4] = {{0., -17. / 60., -5. / 12., 0.}, {0., -15. / 68., -17. / 60., -5. / 12.}};
const double CNRK[2][4] = {{0., 8. / 15., 2. / 3., 0.}, {0., 8. / 17., 8. / 15., 2. / 3.}};

struct Tw {
  double2* d = nullptr;
  float2* f = nullptr;
  FFTPlan plan{};
};

// pieces per state slot in sgpu_offload_steps' copies
#ifndef SB_OFFLOAD_CHUNKS
#define SB_OFFLOAD_CHUNKS 8
#endif
constexpr int OFFLOAD_CHUNKS = SB_OFFLOAD_CHUNKS;

}  // namespace

struct sgpu_ctx {
  sgpu_params prm{};
  Dims g{};
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;      // mean-flow solve, overlapped with the pencils
  cudaEvent_t fork = nullptr, join = nullptr;
  // sgpu_offload_steps: copy streams, per-slot events and per-chunk download
  // events (created on first use)
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t up_done[7] = {}, out_ready[7] = {}, down_done[7 * OFFLOAD_CHUNKS] = {};
  cudaEvent_t ev[16] = {};
  // resident state
  double2* st = nullptr;     // [7][nyp][NP]; SGPU_MIXED keeps only slots 5-6 (p_v, p_omega) here
  float2* stf = nullptr;     // SGPU_MIXED: slots 0-4 (u, v, w, omega_x, omega_z / H) in FP32
  bool mixed = false;
  double* puw = nullptr;     // [2][ny]
  double* scal = nullptr;    // [0] px, [1] mflux
  unsigned long long* cfl_bits = nullptr;
  double* alfa = nullptr;
  double* beta = nullptr;
  double* dyi = nullptr;
  // step-2 buffers
  double2* zb = nullptr;     // [6][nyp][nzp][nx2]
  double2* xb = nullptr;     // [3][nyp][nzp][nx2]
  // step-3 scratch
  double2* cz = nullptr;     // complex scratch columns, [ncz][nyp][NP]
  int ncz = 0;
  double* rz = nullptr;      // real scratch columns, [nrz][nyp][NP]
  int nrz = 0;
  // homogeneous solutions of the three RK stages (k_pencil_hom): v_h
  // [3][nyp][NP], parity sums [3][2 NP], keyed by the stage's a_n + b_n
  double* hom_vh = nullptr;
  double* hom_s = nullptr;
  double* hom_cf = nullptr;  // coefficient columns [3][4][nyp][NP] (k_pencil_hom)
  double hom_key[4] = {0.0, 0.0, 0.0, 0.0};
  int hom_next = 0;
  double* mscr = nullptr;    // mean-flow scratch
  double* meanp = nullptr;   // [4][nyp] U, W, Omega_x, Omega_z for the mixed step 2
  double* ampd = nullptr;    // [20][nyp] plane statistics
  // ADM-RT LES (sgpu_set_les): gu = high-pass filtered u, v, w [3][nyp][NP]
  int iles = 0, les_mode = 2, les_iord = 5;
  double les_chi = 0.0;
  double2* les_gu = nullptr;
  int les_gu_n = 0;            // fields les_gu holds: 3, or 5 for the HPF model (u, v, w, omega_x, omega_z)
  // dynamic HPF model (iles = 3, cs = 0): the secondary filter's x/z tables,
  // the five secondary high-pass filtered fields, and the physical strain of
  // those [6][nyp][nz][nx]
  bool hpf_dyn = false;
  double* les_lpf2 = nullptr;
  double* les_filt2 = nullptr;
  double2* les_gu2 = nullptr;
  double* hpf_s2 = nullptr;
  double* les_coef = nullptr;  // [nyp][LES_ROW]
  double* les_lpf = nullptr;   // [NP] L_xz
  double* les_filt = nullptr;  // [NP] F_xz
  double les_fact2 = 0.0, les_factm2 = 0.0;
  // eddy-viscosity LES (iles = 2): buffers on the unpadded nx x nz grid
  SgsBufs sgs{};
  double* sgs_delta2 = nullptr;  // [nyp] Delta^2 (bla/preprbl.f:62-71)
  double les_cs = 0.0;
  int les_ineg = 1;
  // learned SGS model (sgpu_set_sgs_mlp; internal iles = 4)
  unsigned char* mlp_image = nullptr;
  double* mlp_tau = nullptr;  // [6][nyp][nz][nx] physical tau
  int* mlp_err = nullptr;
  float mlp_s_in = 1.f, mlp_s_y = 1.f, mlp_s_out = 1.f;
  // per-plane fallback of the learned model to the eddy-viscosity model
  // (sgpu_set_sgs_fallback): plane switches [nyp] and the two backscatter sums
  // per plane [2 nyp] of the last evaluation
  bool sgs_fb = false;
  double sgs_fb_bound = 0.0;
  int* sgs_flags = nullptr;
  double* sgs_bsums = nullptr;
  // mixed path: Chebyshev transform matrices for the tensor cores (cheb_tc.cuh)
  unsigned char* chb_fwd = nullptr;  // forward, scale 1/(nxp nzp)
  unsigned char* chb_inv = nullptr;  // inverse
  int* chb_err = nullptr;
  double* stage = nullptr;   // host<->device staging (split re/im)
  Tw twz, twx, twy;
  Tw sgs_twz, sgs_twx;  // lengths nz and nx (iles = 2)
  // xy statistics (sgpu_xys_sample): running sums xys [96][nyp][nx] and
  // sumw, the 15 spectral fields, the z-group sums and physical u
  double* xys = nullptr;
  double2* xys_spec = nullptr;
  double* xys_part = nullptr;
  double* xys_u = nullptr;
  double xys_sumw = 0.0;
  Tw xys_twz, xys_twx;
  float* box_out = nullptr;  // sgpu_box_filter_sample: features then targets
  double2* press = nullptr;     // sgpu_pressure: p [nyp][NP] (Fourier x/z, physical y)
  bool press_valid = false;     // press belongs to the current state
  double* press_wd = nullptr;   // [2][nyp] second-derivative weights at y = +1, -1
  size_t box_n = 0;          // coarse points box_out holds
  // spatial simulation (sgpu_set_fringe, sgpu_set_base_flow): the fringe
  // function at the nxp x points and the base flow [3][nyp][nxp] in physical
  // space, which the fringe damps towards
  double* fr_lam = nullptr;
  double* fr_base = nullptr;
  bool fringe = false;
  // RK bookkeeping (host mirror of the reference driver scalars)
  double an = 0, bn = 0, anp1 = 0, bnp1 = 0, cnp1 = 0, dtn = 0, t = 0, tc = 0;
  // the next full step's time step (the reference's dtnp1, bla/bla.f:2358-2372),
  // set by sgpu_set_dt; equal to dtn for a fixed time step
  double dt_next = 0;
  int it = 1;
  double cfl = 0.0;
  bool cfl_pending = false;
  bool have_state = false;
  long long launches = 0;
  // threads per CTA of the FFT kernels (measured on B200: 256 everywhere but
  // the FP64 x-pass, whose register use prefers 128)
  // rb: z rows per CTA of the FP64 x pass; two (the H3 of both rows paired in
  // one complex FFT, 72 registers, two CTAs of 448 threads per SM) measured
  // 2.24 -> 2.43 ms at 384x193x384
#ifndef SB_XPASS64_RB
#define SB_XPASS64_RB 1
#endif
  static constexpr int kb = 4, rb = SB_XPASS64_RB, pb = 4, fft_threads = 256, xpass64_threads = 128;
  static constexpr int kbf = MIXED_KB, rbf = MIXED_RB, pbf = 8;  // FP32 tiles (mixed.h)
  // optional per-kernel timing (sgpu_profile): event pairs around each launch
  bool prof = false;
  // step 3 with one warp per pencil (pencil_warp.cuh) instead of one thread
  // per pencil (k_pencil); SIMSON_PENCIL_WARP=0/1 overrides the default
  bool pencil_warp = false;
  // bounded waits of the tensor-core kernels (sgpu_set_wait_limit)
  int wait_limit = 0;
  int test_timeout = 0;
  // CUDA graph of one whole RK3 step (sgpu_step_rk), replayed while the step's
  // launch pattern stays the same
  cudaGraphExec_t step_exec = nullptr;
  bool step_valid = false;
  unsigned step_key = 0;         // CFL substep mask, LES mode and pencil kernel of the captured step
  double step_dt = 0.0;          // time step of the captured step
  long long step_launches = 0;   // kernels one captured step launches
  bool graphs = true;
  std::vector<cudaEvent_t> pev;
  std::vector<int> pid;
  int pnext = 0;
};

// the warp-per-pencil step 3 up to this many pencils (auto selection)
constexpr int kPencilWarpMaxPencils = 8192;

enum KernelId { K_ZINV = 0, K_XPASS, K_ZFWD, K_CHEB_FWD, K_PENCIL, K_MEAN, K_CHEB_INV, K_OTHER, K_COUNT };

// NVTX range over a host scope (phases of the step for nsys / ncu --nvtx;
// no-ops unless a tool is attached)
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

static void prof_mark(sgpu_ctx* c, int id) {
  if (!c->prof) return;
  if (c->pnext + 1 >= (int)c->pev.size()) return;
  cudaEventRecord(c->pev[c->pnext], c->stream);
  c->pid[c->pnext] = id;
  c->pnext++;
}

// the fringe arguments of the x passes (none unless sgpu_set_fringe enabled it)
static Fringe ctx_fringe(const sgpu_ctx* c) {
  return c->fringe ? Fringe{c->fr_lam, c->fr_base} : Fringe{nullptr, nullptr};
}

static int cuda_fail(cudaError_t e, const char* where) {
  if (e != cudaSuccess) {
    fprintf(stderr, "simson_b200: %s: %s\n", where, cudaGetErrorString(e));
    return SGPU_E_CUDA;
  }
  return SGPU_OK;
}
#define CK(x)                                        \
  do {                                               \
    int _r = cuda_fail((x), #x);                     \
    if (_r) return _r;                               \
  } while (0)


static int make_tw(Tw& t, int n) {
  t.plan = fft_make_plan(n);
  if (t.plan.npass < 0) return SGPU_E_PARAM;
  std::vector<double2> hd(n);
  std::vector<float2> hf(n);
  for (int m = 0; m < n; ++m) {
    long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
    hd[m] = double2{(double)cosl(ang), (double)sinl(ang)};
    hf[m] = float2{(float)cosl(ang), (float)sinl(ang)};
  }
  CK(cudaMalloc(&t.d, n * sizeof(double2)));
  CK(cudaMalloc(&t.f, n * sizeof(float2)));
  CK(cudaMemcpy(t.d, hd.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(t.f, hf.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
  return SGPU_OK;
}

// ---------------------------------------------------------------------------
// layout conversion between the reference's split arrays and the device state
// ---------------------------------------------------------------------------
// s0: state slot of the first reference slot (re, im point at that slot)
__global__ void k_from_ref(const double* __restrict__ re, const double* __restrict__ im, double2* __restrict__ st,
                           Dims g, int nslots, int s0 = 0) {
  const size_t tot = (size_t)nslots * g.nyp * g.NP;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    // i indexes the reference layout x + nx2*(y + nyp*(z + nz*s))
    size_t r = i;
    const int x = r % g.nx2; r /= g.nx2;
    const int y = r % g.nyp; r /= g.nyp;
    const int z = r % g.nz; r /= g.nz;
    const int s = s0 + (int)r;
    st[((size_t)s * g.nyp + y) * g.NP + (size_t)z * g.nx2 + x] = double2{re[i], im[i]};
  }
}

__global__ void k_to_ref(const double2* __restrict__ st, double* __restrict__ re, double* __restrict__ im, Dims g,
                         int nslots, int s0 = 0) {
  const size_t tot = (size_t)nslots * g.nyp * g.NP;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    size_t r = i;
    const int x = r % g.nx2; r /= g.nx2;
    const int y = r % g.nyp; r /= g.nyp;
    const int z = r % g.nz; r /= g.nz;
    const int s = s0 + (int)r;
    const double2 v = st[((size_t)s * g.nyp + y) * g.NP + (size_t)z * g.nx2 + x];
    re[i] = v.x;
    im[i] = v.y;
  }
}

// SGPU_MIXED: slots 0-4 live in FP32 (stf), slots 5-6 in FP64 (st)
__global__ void k_from_ref_mixed(const double* __restrict__ re, const double* __restrict__ im,
                                 double2* __restrict__ st, float2* __restrict__ stf, Dims g, int nslots,
                                 int s0 = 0) {
  const size_t tot = (size_t)nslots * g.nyp * g.NP;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    size_t r = i;
    const int x = r % g.nx2; r /= g.nx2;
    const int y = r % g.nyp; r /= g.nyp;
    const int z = r % g.nz; r /= g.nz;
    const int s = s0 + (int)r;
    const size_t o = ((size_t)s * g.nyp + y) * g.NP + (size_t)z * g.nx2 + x;
    // every slot also lands in FP64: sgpu_prhs differentiates u, v, w up to
    // four times in y, which FP32 rounding would not survive
    if (s < 5) stf[o] = float2{(float)re[i], (float)im[i]};
    st[o] = double2{re[i], im[i]};
  }
}

__global__ void k_to_ref_mixed(const double2* __restrict__ st, const float2* __restrict__ stf,
                               double* __restrict__ re, double* __restrict__ im, Dims g, int nslots, int s0 = 0) {
  const size_t tot = (size_t)nslots * g.nyp * g.NP;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot; i += (size_t)gridDim.x * blockDim.x) {
    size_t r = i;
    const int x = r % g.nx2; r /= g.nx2;
    const int y = r % g.nyp; r /= g.nyp;
    const int z = r % g.nz; r /= g.nz;
    const int s = s0 + (int)r;
    const size_t o = ((size_t)s * g.nyp + y) * g.NP + (size_t)z * g.nx2 + x;
    if (s < 5) {
      const float2 v = stf[o];
      re[i] = (double)v.x;
      im[i] = (double)v.y;
    } else {
      const double2 v = st[o];
      re[i] = v.x;
      im[i] = v.y;
    }
  }
}

__global__ void k_cfl_reset(unsigned long long* c) { *c = 0ull; }

// ---------------------------------------------------------------------------

extern "C" const char* sgpu_error_string(int code) {
  switch (code) {
    case SGPU_OK: return "ok";
    case SGPU_E_PARAM: return "invalid parameters";
    case SGPU_E_CUDA: return "CUDA error";
    case SGPU_E_STATE: return "call out of order";
    case SGPU_E_CFL: return "CFL*dt above 10";
    case SGPU_E_NAN: return "non-finite state";
    case SGPU_E_TIMEOUT: return "a bounded device wait ran out";
    default: return "unknown error";
  }
}

static size_t smem_fft(int n, int cols, size_t elem) { return 2 * (size_t)n * cols * elem; }

extern "C" int sgpu_init(const sgpu_params* prm, sgpu_ctx** out) {
  if (!prm || !out) return SGPU_E_PARAM;
  *out = nullptr;
  const sgpu_params& P = *prm;
  if (P.nx < 4 || P.nz < 4 || P.nx % 4 || P.nz % 2 || P.ny < 9 || (P.ny % 2) == 0 || (P.nst != 3 && P.nst != 4) || !(P.dt > 0) ||
      !(P.re > 0) || !(P.xl > 0) || !(P.zl > 0) || (P.precision != SGPU_FP64 && P.precision != SGPU_MIXED))
    return SGPU_E_PARAM;
  sgpu_ctx* c = new sgpu_ctx();
  c->prm = P;
  c->mixed = (P.precision == SGPU_MIXED);
  Dims& g = c->g;
  g.nx = P.nx; g.ny = P.ny; g.nz = P.nz;
  g.nx2 = P.nx / 2; g.nyp = P.ny;
  g.nxp = P.nx + P.nx / 2; g.nzp = P.nz + P.nz / 2;
  g.NP = P.nz * g.nx2; g.zodd = P.nz / 2;
  g.y0 = 0; g.y1 = g.nyp; g.p0 = 0; g.p1 = g.NP;  // the whole domain
  int rc = SGPU_OK;
  auto fail = [&](int r) { sgpu_finalize(c); return r; };
  if (cudaSetDevice(P.device) != cudaSuccess) return fail(SGPU_E_CUDA);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(SGPU_E_CUDA);
  // the mean-flow block goes on a high-priority stream: launched at the same
  // time as the pencil grid (one full wave), it must be placed first, or it
  // waits for the whole wave to retire and the overlap is lost
  int prio_lo = 0, prio_hi = 0;
  if (cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi) != cudaSuccess) return fail(SGPU_E_CUDA);
  if (cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_hi) != cudaSuccess)
    return fail(SGPU_E_CUDA);
  if (cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming) != cudaSuccess)
    return fail(SGPU_E_CUDA);
  for (int i = 0; i < 16; ++i)
    if (cudaEventCreate(&c->ev[i]) != cudaSuccess) return fail(SGPU_E_CUDA);
  if ((rc = make_tw(c->twz, g.nzp)) || (rc = make_tw(c->twx, g.nxp)) || (rc = make_tw(c->twy, 2 * (g.nyp - 1))))
    return fail(rc);
  const size_t fld = (size_t)g.nyp * g.NP;
  c->ncz = 21;  // complex scratch fields czf(c, 0..20)
  c->nrz = 2;
  if (cudaMalloc(&c->st, 7 * fld * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&c->puw, 2 * g.ny * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->scal, 4 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->cfl_bits, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&c->alfa, g.nx2 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->beta, g.nz * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->dyi, g.nyp * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->zb, 6 * (size_t)g.nyp * g.nzp * g.nx2 * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&c->xb, 3 * (size_t)g.nyp * g.nzp * g.nx2 * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&c->cz, (size_t)c->ncz * fld * sizeof(double2)) != cudaSuccess ||
      cudaMalloc(&c->rz, (size_t)c->nrz * fld * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->mscr, 16 * (size_t)g.nyp * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->hom_vh, (size_t)P.nst * fld * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->hom_s, (size_t)P.nst * 2 * (size_t)g.NP * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->hom_cf, (size_t)P.nst * 4 * fld * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->stage, 2 * 7 * fld * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->ampd, 20 * (size_t)g.nyp * sizeof(double)) != cudaSuccess)
    return fail(SGPU_E_CUDA);
  if (c->mixed && (cudaMalloc(&c->stf, 5 * fld * sizeof(float2)) != cudaSuccess ||
                   cudaMalloc(&c->meanp, 4 * (size_t)g.nyp * sizeof(double)) != cudaSuccess))
    return fail(SGPU_E_CUDA);
  if (c->mixed && g.nyp <= CHB_MAX_NY) {
    // the step's two Chebyshev transforms as tensor-core GEMMs (up to
    // CHB_MAX_NY points in y; larger grids keep the FFT transforms)
    std::vector<unsigned char> mf, mi;
    chb_build_matrix(g.nyp, 0, 1.0 / ((double)g.nxp * (double)g.nzp), mf);
    chb_build_matrix(g.nyp, 1, 1.0, mi);
    if (cudaMalloc(&c->chb_fwd, mf.size()) != cudaSuccess || cudaMalloc(&c->chb_inv, mi.size()) != cudaSuccess ||
        cudaMalloc(&c->chb_err, sizeof(int)) != cudaSuccess)
      return fail(SGPU_E_CUDA);
    cudaMemcpy(c->chb_fwd, mf.data(), mf.size(), cudaMemcpyHostToDevice);
    cudaMemcpy(c->chb_inv, mi.data(), mi.size(), cudaMemcpyHostToDevice);
    cudaMemset(c->chb_err, 0, sizeof(int));
    cudaFuncSetAttribute(k_cheb_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, CHB_SMEM);
  }
  cudaMemset(c->st, 0, 7 * fld * sizeof(double2));
  cudaMemset(c->puw, 0, 2 * g.ny * sizeof(double));
  // wavenumbers (bla/preprbl.f:36-43) and CFL grid spacing (bla/boxcfl.f:25-56)
  const double pi = 3.1415926535897932385;
  std::vector<double> alfa(g.nx2), beta(g.nz, 0.0), dyi(g.nyp), eta(g.nyp), deta(g.nyp);
  for (int x = 0; x < g.nx2; ++x) alfa[x] = 2. * pi / P.xl * (double)x;
  for (int z = 1; z <= g.nz / 2; ++z) {
    beta[z] = 2. * pi / P.zl * (double)z;
    beta[g.nz - z] = -2. * pi / P.zl * (double)z;
  }
  for (int y = 0; y < g.nyp; ++y) eta[y] = cos(pi * (double)y / (double)(g.nyp - 1));
  deta[0] = 1. - eta[1];
  deta[g.nyp - 1] = deta[0];
  for (int y = 1; y < g.nyp - 1; ++y) deta[y] = (eta[y - 1] - eta[y + 1]) * .5;
  for (int y = 0; y < g.nyp; ++y) {
    double d = (double)(g.ny - 1) / (double)(g.nyp - 1) / deta[y];
    if (g.ny >= 17) d = fmin(d, (double)(g.ny - 1) * (double)(g.ny - 1) / 10. / 3.14);
    dyi[y] = d;
  }
  cudaMemcpy(c->alfa, alfa.data(), g.nx2 * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(c->beta, beta.data(), g.nz * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(c->dyi, dyi.data(), g.nyp * sizeof(double), cudaMemcpyHostToDevice);
  double sc[4] = {P.px, P.mflux, 0, 0};
  cudaMemcpy(c->scal, sc, sizeof(sc), cudaMemcpyHostToDevice);
  // shared-memory opt-in
  const size_t s_z = smem_fft(g.nzp, c->kb, sizeof(double2));
  const size_t s_x = smem_fft(g.nxp, 3 * c->rb, sizeof(double2));
  const size_t s_y = smem_fft(2 * (g.nyp - 1), c->pb, sizeof(double2));
  const size_t s_zf = smem_fft(g.nzp, sgpu_ctx::kbf, sizeof(float2));
  const size_t s_xf = smem_fft(g.nxp, 3 * sgpu_ctx::rbf, sizeof(float2));
  const size_t s_yf = smem_fft(2 * (g.nyp - 1), sgpu_ctx::pbf, sizeof(float2));
  if (s_z > 227 * 1024 || s_x > 227 * 1024 || s_y > 227 * 1024 || s_zf > 227 * 1024 || s_xf > 227 * 1024 ||
      s_yf > 227 * 1024)
    return fail(SGPU_E_PARAM);
  cudaFuncSetAttribute(k_cheb<double, sgpu_ctx::pb, double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)s_y);
  // FP32 variants (their own tiles)
  cudaFuncSetAttribute(k_cheb<float, sgpu_ctx::pbf, float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)s_yf);
  cudaFuncSetAttribute(k_cheb<float, sgpu_ctx::pbf, double, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)s_yf);
  cudaFuncSetAttribute(k_cheb<float, sgpu_ctx::pbf, float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)s_yf);
  c->dtn = P.dt;
  c->dt_next = P.dt;
  // SIMSON_GRAPHS=0: launch every kernel directly (no CUDA-graph replay)
  const char* ge = getenv("SIMSON_GRAPHS");
  c->graphs = !(ge && ge[0] == '0');
  // step 3's pencil kernel: one warp per pencil on grids with few pencils
  // (its parallelism is per pencil: 0.11 against 0.42 ms at 64x97x64, 2 048
  // pencils; 0.28 against 0.58 ms at 96x129x96, 4 608), one thread per
  // pencil on large grids (0.58 against 0.85 ms at 192x129x160, 15 360; 1.3
  // against 5.2 ms at 384x193x384, 73 728, where the thread kernel streams
  // near the DRAM bandwidth); SIMSON_PENCIL_WARP=0/1 forces one of them
  const char* pw = getenv("SIMSON_PENCIL_WARP");
  c->pencil_warp = pencil_warp_rows(g.nyp) > 0 && (pw ? pw[0] == '1' : g.NP <= kPencilWarpMaxPencils);
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(SGPU_E_CUDA);
  *out = c;
  return SGPU_OK;
}

extern "C" int sgpu_finalize(sgpu_ctx* c) {
  if (!c) return SGPU_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->step_exec) cudaGraphExecDestroy(c->step_exec);
  void* ptrs[] = {c->st, c->stf, c->meanp, c->ampd, c->les_gu, c->les_coef, c->les_lpf, c->les_filt,
                  c->sgs.spec9, c->sgs.phys10, c->sgs.filt21, c->sgs.numden, c->sgs.cxy, c->sgs.tauz6, c->sgs.tau,
                  c->sgs_delta2, c->sgs_twz.d, c->sgs_twz.f, c->sgs_twx.d, c->sgs_twx.f, c->xys, c->xys_spec,
                  c->xys_part, c->xys_u, c->box_out, c->press, c->press_wd, c->xys_twz.d, c->xys_twz.f, c->xys_twx.d, c->xys_twx.f, c->mlp_image, c->mlp_tau,
                  c->mlp_err, c->sgs_flags, c->sgs_bsums, c->chb_fwd, c->chb_inv, c->chb_err, c->puw, c->scal, c->cfl_bits, c->alfa, c->beta, c->dyi, c->zb, c->xb, c->cz, c->rz,
                  c->mscr, c->hom_vh, c->hom_s, c->hom_cf, c->stage, c->twz.d, c->twz.f, c->twx.d, c->twx.f, c->twy.d, c->twy.f,
                  c->fr_lam, c->fr_base, c->les_lpf2, c->les_filt2, c->les_gu2, c->hpf_s2};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int i = 0; i < 16; ++i)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  for (auto& e : c->pev) cudaEventDestroy(e);
  if (c->fork) cudaEventDestroy(c->fork);
  if (c->join) cudaEventDestroy(c->join);
  for (int k = 0; k < 7; ++k) {
    if (c->up_done[k]) cudaEventDestroy(c->up_done[k]);
    if (c->out_ready[k]) cudaEventDestroy(c->out_ready[k]);
  }
  for (auto& e : c->down_done)
    if (e) cudaEventDestroy(e);
  if (c->h2d) cudaStreamDestroy(c->h2d);
  if (c->d2h) cudaStreamDestroy(c->d2h);
  if (c->side) cudaStreamDestroy(c->side);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SGPU_OK;
}

extern "C" int sgpu_upload_state(sgpu_ctx* c, const double* ur, const double* ui, int nslots) {
  if (c) c->press_valid = false;  // the state changes
  if (!c || !ur || !ui || nslots < 1 || nslots > 7) return SGPU_E_PARAM;
  const size_t n = (size_t)nslots * c->g.nyp * c->g.NP;
  CK(cudaMemcpyAsync(c->stage, ur, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->stage + n, ui, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (c->mixed)
    k_from_ref_mixed<<<592, 256, 0, c->stream>>>(c->stage, c->stage + n, c->st, c->stf, c->g, nslots);
  else
    k_from_ref<<<592, 256, 0, c->stream>>>(c->stage, c->stage + n, c->st, c->g, nslots);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  c->have_state = true;
  return SGPU_OK;
}

extern "C" int sgpu_download_state(sgpu_ctx* c, double* ur, double* ui, int nslots) {
  if (!c || !ur || !ui || nslots < 1 || nslots > 7) return SGPU_E_PARAM;
  const size_t n = (size_t)nslots * c->g.nyp * c->g.NP;
  if (c->mixed)
    k_to_ref_mixed<<<592, 256, 0, c->stream>>>(c->st, c->stf, c->stage, c->stage + n, c->g, nslots);
  else
    k_to_ref<<<592, 256, 0, c->stream>>>(c->st, c->stage, c->stage + n, c->g, nslots);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(ur, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(ui, c->stage + n, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

extern "C" int sgpu_upload_puw(sgpu_ctx* c, const double* puw) {
  if (!c || !puw) return SGPU_E_PARAM;
  CK(cudaMemcpyAsync(c->puw, puw, 2 * c->g.ny * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

extern "C" int sgpu_download_puw(sgpu_ctx* c, double* puw) {
  if (!c || !puw) return SGPU_E_PARAM;
  CK(cudaMemcpyAsync(puw, c->puw, 2 * c->g.ny * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

static double2* czf(sgpu_ctx* c, int k) { return c->cz + (size_t)k * c->g.nyp * c->g.NP; }
static double* rzf(sgpu_ctx* c, int k) { return c->rz + (size_t)k * c->g.nyp * c->g.NP; }
static double2* slot(sgpu_ctx* c, int s) { return c->st + (size_t)s * c->g.nyp * c->g.NP; }

template <class T, int PB, class SI, class SO>
static void launch_cheb_t(sgpu_ctx* c, const typename C2<SI>::type* in, size_t in_fs, typename C2<SO>::type* out,
                          size_t out_fs, int nfields, int inverse, double scale, int skip_oddball,
                          const typename C2<T>::type* tw) {
  const Dims& g = c->g;
  dim3 grid((g.p1 - g.p0 + PB - 1) / PB, nfields);
  const size_t sm = smem_fft(2 * (g.nyp - 1), PB, sizeof(typename C2<T>::type));
  // transform lengths 2(ny-1) of the production and test grids take the
  // compile-time plan
  switch (2 * (g.nyp - 1)) {
#define SB_CHEB_CASE(L)                                                                                      \
  case L: {                                                                                                  \
    constexpr int NT = fixed_threads(L, PB);                                                                 \
    cudaFuncSetAttribute(k_cheb<T, PB, SI, SO, L, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
    k_cheb<T, PB, SI, SO, L, NT><<<grid, NT, sm, c->stream>>>(in, in_fs, out, out_fs, g, inverse, scale,      \
                                                              c->twy.plan, tw, skip_oddball);               \
    break;                                                                                                   \
  }
    SB_CHEB_CASE(128) SB_CHEB_CASE(192) SB_CHEB_CASE(256) SB_CHEB_CASE(384)
#undef SB_CHEB_CASE
    default:
      k_cheb<T, PB, SI, SO><<<grid, sgpu_ctx::fft_threads, sm, c->stream>>>(in, in_fs, out, out_fs, g, inverse,
                                                                            scale, c->twy.plan, tw, skip_oddball);
  }
  c->launches++;
}

// Chebyshev transform of nfields y-pencil fields.  Physical-y fields live in
// the state (FP64, or FP32 under SGPU_MIXED); Chebyshev-y fields are FP64.
// Mixed path: the FP32 transforms as a 3xTF32 tensor-core GEMM over all
// pencils (cheb_tc.cuh); fields are float2 arrays seen as 2 NP float columns.
static void launch_cheb_tc(sgpu_ctx* c, const float2* in, size_t in_fs, float2* out, size_t out_fs, int nfields,
                           const unsigned char* mat, int skip_oddball) {
  const Dims& g = c->g;
  ChebTCArgs A{};
  // this context's pencils p0 <= p < p1 (columns 2 p0 .. 2 p1 of the full fields)
  A.in = reinterpret_cast<const float*>(in) + 2 * (size_t)g.p0;
  A.in_fs = 2 * in_fs;
  A.out = reinterpret_cast<float*>(out) + 2 * (size_t)g.p0;
  A.out_fs = 2 * out_fs;
  A.ncol = 2 * (g.p1 - g.p0);
  A.ld = 2 * g.NP;
  A.p0 = g.p0;
  A.n = g.nyp;
  A.inverse = (mat == c->chb_inv) ? 1 : 0;
  A.ne = chb_even_chunks(g.nyp);
  A.no = chb_odd_chunks(g.nyp);
  const int H = (g.nyp - 1) / 2;
  A.nre = (H + 1 + 15) / 16 * 16;
  A.nro = (H + 15) / 16 * 16;
  A.mat = mat;
  A.skip_oddball = skip_oddball;
  A.nx2 = g.nx2;
  A.zodd = g.zodd;
  A.err = c->chb_err;
  A.wait_limit = c->wait_limit;
  A.test_timeout = c->test_timeout;
  dim3 grid((A.ncol + CHB_TILE - 1) / CHB_TILE, nfields);
  k_cheb_tc<<<grid, CHB_THREADS, CHB_SMEM, c->stream>>>(A);
  c->launches++;
}

static void cheb_to_spec(sgpu_ctx* c, int slot0, double2* out, int nfields, double scale) {
  const size_t fld = (size_t)c->g.nyp * c->g.NP;
  const double step_scale = 1.0 / ((double)c->g.nxp * (double)c->g.nzp);
  if (c->mixed && c->chb_fwd && scale == step_scale)  // FP32 Chebyshev coefficients of H (read as float2)
    // the output fields sit where the FP64 scratch fields would (stride fld
    // double2 = 2*fld float2), so the pencil kernel addresses them as usual;
    // the prepared matrix carries the step's scale 1/(nxp nzp)
    launch_cheb_tc(c, c->stf + slot0 * fld, fld, reinterpret_cast<float2*>(out), 2 * fld, nfields, c->chb_fwd, 0);
  else if (c->mixed)
    launch_cheb_t<float, sgpu_ctx::pbf, float, float>(c, c->stf + slot0 * fld, fld, reinterpret_cast<float2*>(out),
                                                      2 * fld, nfields, 0, scale, 0, c->twy.f);
  else
    launch_cheb_t<double, sgpu_ctx::pb, double, double>(c, c->st + slot0 * fld, fld, out, fld, nfields, 0, scale, 0,
                                                        c->twy.d);
}

static void cheb_to_phys(sgpu_ctx* c, const double2* in, int slot0, int nfields, int skip_oddball,
                         bool fp32_input = false) {
  const size_t fld = (size_t)c->g.nyp * c->g.NP;
  if (c->mixed && fp32_input && c->chb_inv)
    launch_cheb_tc(c, reinterpret_cast<const float2*>(in), 2 * fld, c->stf + slot0 * fld, fld, nfields, c->chb_inv,
                   skip_oddball);
  else if (c->mixed && fp32_input)
    launch_cheb_t<float, sgpu_ctx::pbf, float, float>(c, reinterpret_cast<const float2*>(in), 2 * fld,
                                                      c->stf + slot0 * fld, fld, nfields, 1, 1.0, skip_oddball,
                                                      c->twy.f);
  else if (c->mixed)
    launch_cheb_t<float, sgpu_ctx::pbf, double, float>(c, in, fld, c->stf + slot0 * fld, fld, nfields, 1, 1.0,
                                                       skip_oddball, c->twy.f);
  else
    launch_cheb_t<double, sgpu_ctx::pb, double, double>(c, in, fld, c->st + slot0 * fld, fld, nfields, 1, 1.0,
                                                        skip_oddball, c->twy.d);
}

static void les_filter_velocity(sgpu_ctx* c, int skip_oddball);

static bool sharded(const sgpu_ctx* c) {
  const Dims& g = c->g;
  return g.y0 != 0 || g.y1 != g.nyp || g.p0 != 0 || g.p1 != g.NP;
}

// the whole domain for the duration of a call (sgpu_prhs works on every
// pencil in every context: its inputs are the whole uploaded state)
struct WholeDomain {
  sgpu_ctx* c;
  Dims keep;
  explicit WholeDomain(sgpu_ctx* ctx) : c(ctx), keep(ctx->g) {
    c->g.y0 = 0; c->g.y1 = c->g.nyp; c->g.p0 = 0; c->g.p1 = c->g.NP;
  }
  ~WholeDomain() { c->g = keep; }
};

extern "C" int sgpu_set_shard(sgpu_ctx* c, int ylo, int yhi, int zlo, int zhi) {
  if (c) c->step_valid = false;  // the captured step no longer matches
  if (!c) return SGPU_E_PARAM;
  const Dims& g = c->g;
  if (ylo < 0 || yhi > g.nyp || ylo >= yhi || zlo < 0 || zhi > g.nz || zlo >= zhi) return SGPU_E_PARAM;
  const bool whole = ylo == 0 && yhi == g.nyp && zlo == 0 && zhi == g.nz;
  if (!whole && c->iles != 0) return SGPU_E_PARAM;  // LES needs the whole domain
  c->g.y0 = ylo; c->g.y1 = yhi;
  c->g.p0 = zlo * g.nx2; c->g.p1 = zhi * g.nx2;
  return SGPU_OK;
}

extern "C" int sgpu_copy_block(sgpu_ctx* c, int slot0, int nslots, int ylo, int yhi, int zlo, int zhi, void* buf,
                               int to_state, size_t* bytes) {
  if (c) c->press_valid = false;  // may write the state
  if (!c || !bytes) return SGPU_E_PARAM;
  const bool nosync = (to_state & SGPU_BLOCK_NOSYNC) != 0;
  to_state &= ~SGPU_BLOCK_NOSYNC;
  if (to_state != 0 && to_state != 1) return SGPU_E_PARAM;
  const Dims& g = c->g;
  if (slot0 < 0 || nslots < 1 || slot0 + nslots > 7 || ylo < 0 || yhi > g.nyp || ylo >= yhi || zlo < 0 ||
      zhi > g.nz || zlo >= zhi)
    return SGPU_E_PARAM;
  const size_t fld = (size_t)g.nyp * g.NP;
  size_t off = 0;
  for (int s = slot0; s < slot0 + nslots; ++s) {
    // complex FP32 under SGPU_MIXED for slots 0-4, complex FP64 otherwise
    const bool f32 = c->mixed && s < 5;
    const size_t es = f32 ? sizeof(float2) : sizeof(double2);
    char* base = f32 ? reinterpret_cast<char*>(c->stf + s * fld) : reinterpret_cast<char*>(c->st + s * fld);
    char* src = base + ((size_t)ylo * g.NP + (size_t)zlo * g.nx2) * es;
    const size_t width = (size_t)(zhi - zlo) * g.nx2 * es, pitch = (size_t)g.NP * es;
    const size_t height = (size_t)(yhi - ylo);
    if (buf) {
      char* b = static_cast<char*>(buf) + off;
      if (to_state)
        CK(cudaMemcpy2DAsync(src, pitch, b, width, width, height, cudaMemcpyDeviceToDevice, c->stream));
      else
        CK(cudaMemcpy2DAsync(b, width, src, pitch, width, height, cudaMemcpyDeviceToDevice, c->stream));
    }
    off += width * height;
  }
  *bytes = off;
  if (buf && !nosync) CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

extern "C" int sgpu_stream(sgpu_ctx* c, void** stream) {
  if (!c || !stream) return SGPU_E_PARAM;
  *stream = static_cast<void*>(c->stream);
  return SGPU_OK;
}

extern "C" int sgpu_prhs(sgpu_ctx* c) {
  if (c) c->press_valid = false;
  NvtxRange nv("prhs");
  if (!c) return SGPU_E_PARAM;
  if (!c->have_state) return SGPU_E_STATE;
  WholeDomain whole(c);
  const Dims& g = c->g;
  const size_t fld = (size_t)g.nyp * g.NP;
  // first-stage RK factors (bla/bla.f:1466-1478) and cflux px (:1622-1633)
  c->dtn = c->dt_next;
  c->an = c->dtn * ANRK[c->prm.nst - 3][0];
  c->cnp1 = 0.0;
  c->anp1 = c->an;
  c->bnp1 = 0.0;
  c->bn = 0.0;
  c->it = 1;
  c->t = 0.0;
  c->tc = 0.0;
  // px and the mass flux of the run's start (bla/bla.f:1622-1633): a restart
  // on the same context does not inherit the last run's values
  const double sc0[4] = {c->prm.px, c->prm.mflux, 0.0, 0.0};
  CK(cudaMemcpyAsync(c->scal, sc0, sizeof(sc0), cudaMemcpyHostToDevice, c->stream));
  // Chebyshev coefficients of u, v, w, from the FP64 copy uploaded with the
  // state (also under SGPU_MIXED: p_v needs four y-derivatives of v)
  launch_cheb_t<double, sgpu_ctx::pb, double, double>(c, c->st, fld, czf(c, 0), fld, 3, 0, 1.0, 0, c->twy.d);
  PrhsBufs B;
  B.U1 = czf(c, 0); B.U2 = czf(c, 1); B.U3 = czf(c, 2);
  B.OMY = czf(c, 3); B.OX = czf(c, 4); B.OZ = czf(c, 5); B.PHI = czf(c, 6); B.T1 = czf(c, 7); B.T2 = czf(c, 8);
  B.PV = slot(c, 5); B.PW = slot(c, 6); B.puw = c->puw;
  k_prhs<<<(g.NP + 127) / 128, 128, 0, c->stream>>>(B, g, c->alfa, c->beta, c->prm.re, c->anp1);
  c->launches++;
  // omega_x, omega_z back to physical y into slots 3, 4
  cheb_to_phys(c, czf(c, 4), 3, 2, 0);
  // ADM-RT: high-pass filtered start-up velocities (bla/prhs.f:95-193)
  if (c->iles == 1 || c->iles == 3) les_filter_velocity(c, 0);
  (void)fld;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

// gu = high-pass filtered u, v, w of the current state (les.cuh); the
// scratch columns are free whenever this runs (after the inverse Chebyshev
// transforms of prhs or of step 3).
static void les_filter_velocity(sgpu_ctx* c, int skip_oddball) {
  const Dims& g = c->g;
  YFilter F{c->les_coef, c->les_fact2, c->les_factm2, g.nyp};
  dim3 grid((g.NP + 127) / 128, c->iles == 3 ? 5 : 3);
  prof_mark(c, K_OTHER);
  if (c->mixed)
    k_les_hpf<float2><<<grid, 128, 0, c->stream>>>(c->stf, c->les_gu, czf(c, 0), F, c->les_lpf, c->les_filt, g,
                                                   c->les_mode, c->les_iord, skip_oddball);
  else
    k_les_hpf<double2><<<grid, 128, 0, c->stream>>>(c->st, c->les_gu, czf(c, 0), F, c->les_lpf, c->les_filt, g,
                                                    c->les_mode, c->les_iord, skip_oddball);
  c->launches++;
  if (c->iles == 3 && c->hpf_dyn) {
    // the secondary filter (bla/linearbl.f:2067-2250, the same wall-normal
    // filter, the x/z tables of the quarter cut-off) for the dynamic procedure
    if (c->mixed)
      k_les_hpf<float2><<<grid, 128, 0, c->stream>>>(c->stf, c->les_gu2, czf(c, 0), F, c->les_lpf2, c->les_filt2, g,
                                                     c->les_mode, c->les_iord, skip_oddball);
    else
      k_les_hpf<double2><<<grid, 128, 0, c->stream>>>(c->st, c->les_gu2, czf(c, 0), F, c->les_lpf2, c->les_filt2,
                                                      g, c->les_mode, c->les_iord, skip_oddball);
    c->launches++;
  }
}

static SgsGrid sgs_grid(const sgpu_ctx* c) {
  const Dims& g = c->g;
  return SgsGrid{g.nx, g.nz, g.nx2, g.nx / 4, g.nyp, g.NP, g.zodd};
}

// Eddy-viscosity SGS force sigma_i = d tau_ij/dx_j of the current state into
// les_gu (bla/les.f + bla/sgs_stress.f, before nonlinbl in every substep).
static void enqueue_sgs(sgpu_ctx* c) {
  const Dims& g = c->g;
  const SgsGrid G = sgs_grid(c);
  constexpr int KB = 4;
  const size_t sz = 2 * (size_t)g.nz * KB * sizeof(double2);
  const size_t sx11 = 2 * (size_t)g.nx * 11 * sizeof(double2);
  const size_t sx3 = 2 * (size_t)g.nx * 3 * sizeof(double2);
  prof_mark(c, K_OTHER);
  dim3 gz((g.nx2 + KB - 1) / KB, g.nyp), gz4((G.nx4 + KB - 1) / KB, g.nyp), gx(g.nz, g.nyp);
  const int set = (c->iles == 4) ? 1 : 0;
  const double* s2 = nullptr;
  if (c->iles == 3 && c->hpf_dyn) {
    // dynamic HPF (bla/les.f:968-1383): first the strain of the secondary
    // filtered field in physical space (test-filtered below in place of S),
    // then u of the state with the strain of the primary filtered field
    k_sgs_zinv<double2, KB><<<gz, 256, sz, c->stream>>>(c->les_gu2, c->sgs, G, c->sgs_twz.plan, c->sgs_twz.d,
                                                        c->alfa, c->beta, 0, nullptr);
    k_sgs_xinv9<<<gx, 128, 2 * (size_t)g.nx * 5 * sizeof(double2), c->stream>>>(c->sgs, G, c->sgs_twx.plan,
                                                                                 c->sgs_twx.d, c->hpf_s2, 3);
    s2 = c->hpf_s2;
    c->launches += 2;
    if (c->mixed)
      k_sgs_zinv<float2, KB><<<gz, 256, sz, c->stream>>>(c->stf, c->sgs, G, c->sgs_twz.plan, c->sgs_twz.d, c->alfa,
                                                         c->beta, 0, c->les_gu);
    else
      k_sgs_zinv<double2, KB><<<gz, 256, sz, c->stream>>>(c->st, c->sgs, G, c->sgs_twz.plan, c->sgs_twz.d, c->alfa,
                                                          c->beta, 0, c->les_gu);
  } else if (c->iles == 3) {
    // HPF model, fixed constant: the strain of the high-pass filtered fields
    // (bla/les.f:404-450, 883-966)
    k_sgs_zinv<double2, KB><<<gz, 256, sz, c->stream>>>(c->les_gu, c->sgs, G, c->sgs_twz.plan, c->sgs_twz.d,
                                                        c->alfa, c->beta, 0, nullptr);
  } else if (c->mixed) {
    k_sgs_zinv<float2, KB><<<gz, 256, sz, c->stream>>>(c->stf, c->sgs, G, c->sgs_twz.plan, c->sgs_twz.d, c->alfa,
                                                       c->beta, set, nullptr);
  } else {
    k_sgs_zinv<double2, KB><<<gz, 256, sz, c->stream>>>(c->st, c->sgs, G, c->sgs_twz.plan, c->sgs_twz.d, c->alfa,
                                                        c->beta, set, nullptr);
  }
  if (c->iles == 4) {
    // learned model: gradients to physical space, MLP on the tensor cores,
    // tau / (nx nz) back to Fourier space
    k_sgs_xinv9<<<gx, 128, 2 * (size_t)g.nx * 5 * sizeof(double2), c->stream>>>(c->sgs, G, c->sgs_twx.plan,
                                                                                 c->sgs_twx.d, c->sgs.phys10, 0);
    MlpArgs A{};
    A.image = c->mlp_image;
    A.mode = 1;
    A.n = (long long)g.nyp * g.nz * g.nx;
    A.grad = c->sgs.phys10;
    A.tau = c->mlp_tau;
    A.plane = g.nz * g.nx;
    A.nyp = g.nyp;
    A.s_in = c->mlp_s_in;
    A.s_y = c->mlp_s_y;
    A.s_out = c->mlp_s_out;
    A.err = c->mlp_err;
    A.wait_limit = c->wait_limit;
    A.test_timeout = c->test_timeout;
    const long long tiles = (A.n + MLP_ROWS - 1) / MLP_ROWS;
    const int blocks = (int)std::min<long long>(tiles, 148 * 4);
    k_sgs_mlp<<<blocks, 128, MLP_SMEM_LAUNCH, c->stream>>>(A);
    c->launches += 2;
    SgsBufs F = c->sgs;
    if (c->sgs_fb) {
      // per-plane fallback: planes whose predicted backscatter exceeds the
      // bound take the eddy-viscosity stress (its kernels skip the others)
      k_sgs_backscatter<<<g.nyp, 1024, 0, c->stream>>>(c->sgs, G, c->mlp_tau, c->sgs_fb_bound, c->sgs_flags,
                                                       c->sgs_bsums);
      F.plane_on = c->sgs_flags;
      if (c->mixed)
        k_sgs_zinv<float2, KB><<<gz, 256, sz, c->stream>>>(c->stf, F, G, c->sgs_twz.plan, c->sgs_twz.d, c->alfa,
                                                           c->beta, 0, nullptr);
      else
        k_sgs_zinv<double2, KB><<<gz, 256, sz, c->stream>>>(c->st, F, G, c->sgs_twz.plan, c->sgs_twz.d, c->alfa,
                                                            c->beta, 0, nullptr);
      k_sgs_xpass1<<<gx, 128, sx11, c->stream>>>(F, G, c->sgs_twx.plan, c->sgs_twx.d, c->sgs_delta2, nullptr);
      k_sgs_zfilt<KB><<<gz4, 256, sz, c->stream>>>(F, G, c->sgs_twz.plan, c->sgs_twz.d);
      k_sgs_xpass2<<<gx, 128, sx11, c->stream>>>(F, G, c->sgs_twx.plan, c->sgs_twx.d, c->sgs_delta2);
      k_sgs_coef<<<dim3((g.nx + 127) / 128, g.nyp), 128, 0, c->stream>>>(F, G, c->les_cs, c->les_ineg);
      c->launches += 6;
    }
    k_sgs_tau_x<<<gx, 128, sx3, c->stream>>>(F, G, c->sgs_twx.plan, c->sgs_twx.d, c->sgs_delta2, c->prm.re,
                                             c->les_ineg, c->mlp_tau);
    k_sgs_zfwd<KB><<<gz, 256, sz, c->stream>>>(c->sgs, G, c->sgs_twz.plan, c->sgs_twz.d);
    c->launches += 3;
  } else {
  k_sgs_xpass1<<<gx, 128, sx11, c->stream>>>(c->sgs, G, c->sgs_twx.plan, c->sgs_twx.d, c->sgs_delta2, s2);
  k_sgs_zfilt<KB><<<gz4, 256, sz, c->stream>>>(c->sgs, G, c->sgs_twz.plan, c->sgs_twz.d);
  k_sgs_xpass2<<<gx, 128, sx11, c->stream>>>(c->sgs, G, c->sgs_twx.plan, c->sgs_twx.d, c->sgs_delta2);
  k_sgs_coef<<<dim3((g.nx + 127) / 128, g.nyp), 128, 0, c->stream>>>(c->sgs, G, c->les_cs, c->les_ineg);
  k_sgs_tau_x<<<gx, 128, sx3, c->stream>>>(c->sgs, G, c->sgs_twx.plan, c->sgs_twx.d, c->sgs_delta2, c->prm.re,
                                           c->les_ineg, nullptr);
  k_sgs_zfwd<KB><<<gz, 256, sz, c->stream>>>(c->sgs, G, c->sgs_twz.plan, c->sgs_twz.d);
  c->launches += 7;
  }
  // sigma on Chebyshev coefficients of tau (sgs_stress.f), back to physical y
  const size_t fld = (size_t)g.nyp * g.NP;
  launch_cheb_t<double, sgpu_ctx::pb, double, double>(c, c->sgs.tau, fld, czf(c, 0), fld, 6, 0, 1.0, 0, c->twy.d);
  k_sgs_sigma<<<(unsigned)(((size_t)g.NP * 32 + 127) / 128), 128, 0, c->stream>>>(czf(c, 0), czf(c, 6), G, c->alfa,
                                                                                c->beta);
  c->launches++;
  launch_cheb_t<double, sgpu_ctx::pb, double, double>(c, czf(c, 6), fld, c->les_gu, fld, 3, 1, 1.0, 0, c->twy.d);
}

static int enqueue_nonlin(sgpu_ctx* c) {
  c->press_valid = false;
  NvtxRange nv("step 2 (nonlinbl)");
  const Dims& g = c->g;
  const sgpu_params& P = c->prm;
  c->tc = c->t + c->cnp1;
  if (c->iles >= 2) enqueue_sgs(c);
  // CFL partial maxima only on the substeps the reference evaluates them
  // (nonlinbl.f: mod(it-1,icfl) == 0); the device word keeps the last one.
  const bool do_cfl = (P.icfl > 0) && ((c->it - 1) % P.icfl == 0);
  if (do_cfl) {
    prof_mark(c, K_OTHER);
    k_cfl_reset<<<1, 1, 0, c->stream>>>(c->cfl_bits);
    c->launches++;
  }
  const int nyl = g.y1 - g.y0;  // this context's xz-planes
  dim3 gz((g.nx2 + c->kb - 1) / c->kb, nyl);
  const size_t s_z = smem_fft(g.nzp, c->kb, sizeof(double2));
  const double dxi = (double)(g.nx - 2) / P.xl;
  const double dzi = (double)(g.nz - 2) / P.zl;
  const size_t s_x = smem_fft(g.nxp, 3 * c->rb, sizeof(double2));
  const size_t s_zf = smem_fft(g.nzp, sgpu_ctx::kbf, sizeof(float2));
  const size_t s_xf = smem_fft(g.nxp, 3 * sgpu_ctx::rbf, sizeof(float2));
  unsigned long long* cflp = do_cfl ? c->cfl_bits : nullptr;
  if (c->mixed) {
    // FP32 transforms and products on the FP32 velocity/vorticity fields
    float2* zbf = reinterpret_cast<float2*>(c->zb);
    float2* xbf = reinterpret_cast<float2*>(c->xb);
    dim3 gzf((g.nx2 + sgpu_ctx::kbf - 1) / sgpu_ctx::kbf, nyl);
    dim3 gxf((g.nzp + sgpu_ctx::rbf - 1) / sgpu_ctx::rbf, nyl);
    // the FFTs carry only the perturbations; the mean profiles enter the
    // products analytically and their mean-mean product in FP64
    prof_mark(c, K_ZINV);
    mixed_mean_profiles(c->stream, c->stf, c->meanp, g);
    mixed_zinv(c->stream, gzf, s_zf, c->stf, zbf, g, c->twz.plan, c->twz.f, c->alfa, c->beta);
    prof_mark(c, K_XPASS);
    mixed_xpass(c->stream, gxf, s_xf, zbf, xbf, g, c->twx.plan, c->twx.f, c->dyi, dxi, dzi, P.rot, cflp, c->meanp,
                ctx_fringe(c));
    prof_mark(c, K_ZFWD);
    mixed_zfwd(c->stream, gzf, s_zf, xbf, c->stf, g, c->twz.plan, c->twz.f, c->meanp, P.rot);
    c->launches++;
  } else {
    prof_mark(c, K_ZINV);
    launch_zinv<double, sgpu_ctx::kb, double>(gz, s_z, c->stream, c->st, c->zb, g, c->twz.plan, c->twz.d, c->alfa,
                                              c->beta, 0);
    dim3 gx((g.nzp + c->rb - 1) / c->rb, nyl);
    prof_mark(c, K_XPASS);
    launch_xpass<double, sgpu_ctx::rb, sgpu_ctx::xpass64_threads>(gx, s_x, c->stream, c->zb, c->xb, g, c->twx.plan,
                                                                  c->twx.d, c->dyi, dxi, dzi, P.rot, cflp, nullptr,
                                                                  ctx_fringe(c));
    prof_mark(c, K_ZFWD);
    launch_zfwd<double, sgpu_ctx::kb, double>(gz, s_z, c->stream, c->xb, c->st, g, c->twz.plan, c->twz.d, nullptr,
                                              0.0);
  }
  c->launches += 3;
  if (c->iles >= 1) {
    // ADM-RT relaxation term -chi gu on H (bla/nonlinbl.f:920-965), or the
    // eddy-viscosity SGS force -sigma (chi = 1, :1011-1048)
    const size_t n3 = 3 * (size_t)g.nyp * g.NP;
    const unsigned nb = (unsigned)((n3 + 255) / 256);
    prof_mark(c, K_OTHER);
    if (c->mixed)
      k_les_relax<float2><<<nb, 256, 0, c->stream>>>(c->stf, c->les_gu, g, c->iles == 1 ? c->les_chi : 1.0);
    else
      k_les_relax<double2><<<nb, 256, 0, c->stream>>>(c->st, c->les_gu, g, c->iles == 1 ? c->les_chi : 1.0);
    c->launches++;
  }
  if (do_cfl) c->cfl_pending = true;
  return cuda_fail(cudaGetLastError(), "nonlin launch");
}

// RK weights of the coming linear step (bla/bla.f:2384-2397); the weights of
// the next step's first stage, formed in a step's last substep, take that
// step's time step dtnp1 (:2358-2372)
static void rk_advance(sgpu_ctx* c) {
  const int nst = c->prm.nst;
  c->an = c->anp1;
  c->bn = c->bnp1;
  const int k = c->it % nst;
  const double dtp = (k == 0) ? c->dt_next : c->dtn;
  c->anp1 = dtp * ANRK[nst - 3][k];
  c->bnp1 = dtp * BNRK[nst - 3][k];
  c->cnp1 = dtp * CNRK[nst - 3][k];
}

// substep counter, time and time step after a linear step
// (bla/bla.f:2598-2610)
static void it_advance(sgpu_ctx* c) {
  c->it += 1;
  if ((c->it - 1) % c->prm.nst == 0) {
    c->t = c->t + c->dtn;
    c->dtn = c->dt_next;
  }
}

static int enqueue_linear(sgpu_ctx* c) {
  NvtxRange nv("step 3 (linearbl)");
  c->press_valid = false;
  const Dims& g = c->g;
  const sgpu_params& P = c->prm;
  rk_advance(c);
  RKc rk{c->an, c->bn, c->anp1, c->bnp1};
  // Chebyshev transform of H, normalised by 1/(nxp nzp) (linearbl.f:262-273)
  prof_mark(c, K_CHEB_FWD);
  cheb_to_spec(c, 0, czf(c, 0), 3, 1.0 / ((double)g.nxp * (double)g.nzp));
  PencilBufs B;
  B.H1 = czf(c, 0); B.H2 = czf(c, 1); B.H3 = czf(c, 2);
  B.PV = slot(c, 5); B.PW = slot(c, 6);
  B.HV = czf(c, 5); B.HOM = czf(c, 6);
  B.PHI = czf(c, 9); B.OM = czf(c, 10); B.V = czf(c, 11); B.DV = czf(c, 12);
  B.OU = czf(c, 16); B.OV = czf(c, 17); B.OW = czf(c, 18); B.OX = czf(c, 19); B.OZ = czf(c, 20);
  B.PHIH = rzf(c, 0); B.DVH = rzf(c, 1);
  // kx = kz = 0 (mean flow, cflux) on the side stream, concurrent with the pencils
  MeanArgs M;
  M.H1 = B.H1; M.H3 = B.H3; M.puw = c->puw; M.scal = c->scal; M.scr = c->mscr;
  M.OU = B.OU; M.OV = B.OV; M.OW = B.OW; M.OX = B.OX; M.OZ = B.OZ; M.PV = B.PV; M.PW = B.PW;
  M.cflux = P.cflux;
  // the mean flow belongs to the context that owns pencil 0 (kz = 0)
  const bool own_mean = g.p0 == 0;
  // the warp kernels of step 3 come with the warp mean-flow solve
  auto mean = [&](cudaStream_t st) {
    if (c->pencil_warp && (c->mixed ? launch_mean_warp<float2>(st, M, g, P.re, rk)
                                    : launch_mean_warp<double2>(st, M, g, P.re, rk)))
      return;
    if (c->mixed)
      mixed_mean(st, M, g, P.re, rk);
    else
      k_mean<double2><<<1, 32, 0, st>>>(M, g, P.re, rk);
  };
  if (!own_mean) {
  } else if (c->prof) {
    prof_mark(c, K_MEAN);
    mean(c->stream);
  } else {
    cudaEventRecord(c->fork, c->stream);
    cudaStreamWaitEvent(c->side, c->fork, 0);
    mean(c->side);
    cudaEventRecord(c->join, c->side);
  }
  if (c->pencil_warp) {
    // one warp per pencil: the homogeneous solutions are columns of its own
    // solves, no per-stage cache
    prof_mark(c, K_PENCIL);
    const bool ok = c->mixed ? mixed_pencil_warp(c->stream, B, g, c->alfa, c->beta, P.re, rk)
                             : launch_pencil_warp<double2, double>(c->stream, B, g, c->alfa, c->beta, P.re, rk);
    if (!ok) return SGPU_E_PARAM;
  } else {
  // this stage's homogeneous solutions, computed on its first use (a key of
  // 0 is never a valid a_n + b_n: dt > 0)
  const double anbn = rk.an + rk.bn;
  int hs = -1;
  for (int s = 0; s < c->prm.nst; ++s)
    if (c->hom_key[s] == anbn) hs = s;
  const size_t fld = (size_t)g.nyp * g.NP;
  if (hs < 0) {
    hs = c->hom_next;
    c->hom_next = (c->hom_next + 1) % c->prm.nst;
    c->hom_key[hs] = anbn;
    prof_mark(c, K_OTHER);
    if (c->mixed)
      mixed_pencil_hom(c->stream, B, g, c->alfa, c->beta, P.re, anbn, c->hom_vh + hs * fld,
                       c->hom_s + hs * 2 * (size_t)g.NP, c->hom_cf + hs * 4 * fld);
    else
      k_pencil_hom<double, double><<<(g.p1 - g.p0 + 127) / 128, 128, 0, c->stream>>>(
          B, g, c->alfa, c->beta, P.re, anbn, c->hom_vh + hs * fld, c->hom_s + hs * 2 * (size_t)g.NP,
          c->hom_cf + hs * 4 * fld);
    c->launches++;
  }
  const double* vhc = c->hom_vh + hs * fld;
  const double* hsc = c->hom_s + hs * 2 * (size_t)g.NP;
  double* cfc = c->hom_cf + hs * 4 * fld;
  prof_mark(c, K_PENCIL);
  if (c->mixed)
    mixed_pencil(c->stream, B, g, c->alfa, c->beta, P.re, rk, vhc, hsc, cfc);
  else
    k_pencil<double2, double, double><<<(g.p1 - g.p0 + 127) / 128, 128, 0, c->stream>>>(B, g, c->alfa, c->beta, P.re, rk,
                                                                                 vhc, hsc, cfc);
  }
  if (!c->prof && own_mean) cudaStreamWaitEvent(c->stream, c->join, 0);
  // u, v, w, omega_x, omega_z back to physical y (slots 0-4), oddball plane untouched
  prof_mark(c, K_CHEB_INV);
  cheb_to_phys(c, B.OU, 0, 5, 1, /*fp32_input=*/c->mixed);
  // ADM-RT and HPF: high-pass filtered new velocities (bla/linearbl.f:1871-2060)
  if (c->iles == 1 || c->iles == 3) les_filter_velocity(c, 1);
  prof_mark(c, K_OTHER);
  c->launches += 2;
  it_advance(c);
  return cuda_fail(cudaGetLastError(), "linear launch");
}

static int collect_cfl(sgpu_ctx* c) {
  if (!c->cfl_pending) return SGPU_OK;
  // a shard holds only its planes' partial maximum: the host all-reduces it
  // (sgpu_cfl_partial, sgpu_cfl_set_global) before the stop test
  if (sharded(c)) return SGPU_OK;
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, c->cfl_bits, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double m;
  memcpy(&m, &bits, sizeof(m));
  const double pi = 3.1415926535897932385;
  c->cfl = (m * pi + 2. * fabs(c->prm.rot)) * c->dtn;  // bla/wcflbl.f:87
  c->cfl_pending = false;
  if (!(c->cfl <= 10.)) return std::isnan(c->cfl) ? SGPU_E_NAN : SGPU_E_CFL;
  return SGPU_OK;
}

extern "C" int sgpu_nonlin(sgpu_ctx* c) {
  if (!c) return SGPU_E_PARAM;
  if (!c->have_state) return SGPU_E_STATE;
  int r = enqueue_nonlin(c);
  if (r) return r;
  return collect_cfl(c);
}

extern "C" int sgpu_linear(sgpu_ctx* c) {
  if (!c) return SGPU_E_PARAM;
  if (!c->have_state) return SGPU_E_STATE;
  return enqueue_linear(c);
}

// The CFL number per unit time step of the current state (bla/getdt.f: the
// step-2 transforms to physical space, bla/boxcfl.f's maximum of
// |u|/dx + |v|/dy + |w|/dz over every plane, times pi, plus 2 |rot|): the
// first time step of a variable-step run is cflmax over this.  The state is
// not changed; the step-2 scratch is.
extern "C" int sgpu_cfl_rate(sgpu_ctx* c, double* rate) {
  if (!c || !rate) return SGPU_E_PARAM;
  if (!c->have_state) return SGPU_E_STATE;
  if (sharded(c) || c->cfl_pending) return SGPU_E_STATE;
  const Dims& g = c->g;
  const sgpu_params& P = c->prm;
  k_cfl_reset<<<1, 1, 0, c->stream>>>(c->cfl_bits);
  const int nyl = g.y1 - g.y0;
  const double dxi = (double)(g.nx - 2) / P.xl;
  const double dzi = (double)(g.nz - 2) / P.zl;
  if (c->mixed) {
    float2* zbf = reinterpret_cast<float2*>(c->zb);
    float2* xbf = reinterpret_cast<float2*>(c->xb);
    dim3 gzf((g.nx2 + sgpu_ctx::kbf - 1) / sgpu_ctx::kbf, nyl);
    dim3 gxf((g.nzp + sgpu_ctx::rbf - 1) / sgpu_ctx::rbf, nyl);
    mixed_mean_profiles(c->stream, c->stf, c->meanp, g);
    mixed_zinv(c->stream, gzf, smem_fft(g.nzp, sgpu_ctx::kbf, sizeof(float2)), c->stf, zbf, g, c->twz.plan, c->twz.f,
               c->alfa, c->beta);
    mixed_xpass(c->stream, gxf, smem_fft(g.nxp, 3 * sgpu_ctx::rbf, sizeof(float2)), zbf, xbf, g, c->twx.plan,
                c->twx.f, c->dyi, dxi, dzi, P.rot, c->cfl_bits, c->meanp, Fringe{nullptr, nullptr});
  } else {
    dim3 gz((g.nx2 + c->kb - 1) / c->kb, nyl);
    dim3 gx((g.nzp + c->rb - 1) / c->rb, nyl);
    launch_zinv<double, sgpu_ctx::kb, double>(gz, smem_fft(g.nzp, c->kb, sizeof(double2)), c->stream, c->st, c->zb,
                                              g, c->twz.plan, c->twz.d, c->alfa, c->beta, 0);
    launch_xpass<double, sgpu_ctx::rb, sgpu_ctx::xpass64_threads>(gx, smem_fft(g.nxp, 3 * c->rb, sizeof(double2)),
                                                                  c->stream, c->zb, c->xb, g, c->twx.plan, c->twx.d,
                                                                  c->dyi, dxi, dzi, P.rot, c->cfl_bits, nullptr,
                                                                  Fringe{nullptr, nullptr});
  }
  c->launches += c->mixed ? 4 : 3;
  CK(cudaGetLastError());
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, c->cfl_bits, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double m;
  memcpy(&m, &bits, sizeof(m));
  const double pi = 3.1415926535897932385;
  *rate = m * pi + 2. * fabs(P.rot);
  return SGPU_OK;
}

// The time step of the next full step (bla/bla.f:2358-2372 dtnp1, applied as
// :2389-2397 and :2610 do).  Before sgpu_prhs: the first step's.
extern "C" int sgpu_set_dt(sgpu_ctx* c, double dt) {
  if (!c || !(dt > 0.0) || !std::isfinite(dt)) return SGPU_E_PARAM;
  c->dt_next = dt;
  return SGPU_OK;
}

// Sharded runs: the partial maximum of this shard's planes, and the stop
// test on the all-reduced one (bla/wcflbl.f:82-98 with MPI_Allreduce).  The
// partial maximum is read only when a substep evaluated it.
extern "C" int sgpu_cfl_partial(sgpu_ctx* c, double* cflp, int* pending) {
  if (!c || !cflp || !pending) return SGPU_E_PARAM;
  *pending = c->cfl_pending ? 1 : 0;
  *cflp = 0.0;
  if (!c->cfl_pending) return SGPU_OK;  // nothing to reduce: no wait
  unsigned long long bits = 0;
  CK(cudaMemcpyAsync(&bits, c->cfl_bits, sizeof(bits), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  memcpy(cflp, &bits, sizeof(double));
  return SGPU_OK;
}

extern "C" int sgpu_cfl_set_global(sgpu_ctx* c, double cflp) {
  if (!c) return SGPU_E_PARAM;
  const double pi = 3.1415926535897932385;
  c->cfl = (cflp * pi + 2. * fabs(c->prm.rot)) * c->dtn;  // bla/wcflbl.f:87
  c->cfl_pending = false;
  if (!(c->cfl <= 10.)) return std::isnan(c->cfl) ? SGPU_E_NAN : SGPU_E_CFL;
  return SGPU_OK;
}

// Launch pattern of the RK step that starts now: bits 0-3 the substeps that
// evaluate the CFL number, bits 4-7 the LES mode, bit 8 the pencil kernel,
// bit 9 the fringe.
// 0xffffffff: the step cannot be replayed (not at a step boundary, its time
// step changes at its end, or a stage's homogeneous solutions not yet
// cached: that substep launches k_pencil_hom).
static unsigned step_pattern(const sgpu_ctx* c) {
  const int nst = c->prm.nst;
  if ((c->it - 1) % nst != 0 || c->dt_next != c->dtn) return 0xffffffffu;
  unsigned key = ((unsigned)c->iles << 4) | ((c->pencil_warp ? 1u : 0u) << 8) | ((c->fringe ? 1u : 0u) << 9);
  double anp1 = c->anp1, bnp1 = c->bnp1;
  for (int s = 0; s < nst; ++s) {
    const int it = c->it + s;
    if (c->prm.icfl > 0 && (it - 1) % c->prm.icfl == 0) key |= 1u << s;
    const double anbn = anp1 + bnp1;  // a_n + b_n of this substep's linear step
    bool cached = c->pencil_warp;  // the warp kernel keeps no per-stage cache
    for (int h = 0; h < nst; ++h) cached = cached || c->hom_key[h] == anbn;
    if (!cached) return 0xffffffffu;
    anp1 = c->dtn * ANRK[nst - 3][it % nst];
    bnp1 = c->dtn * BNRK[nst - 3][it % nst];
  }
  return key;
}

// Capture the substeps of this step into c->step_exec (launching nothing);
// the host bookkeeping advances as in a direct launch.  On failure the host
// state is restored and the caller launches directly.
static int capture_step(sgpu_ctx* c, unsigned key) {
  NvtxRange nv("capture RK step");
  const double an = c->an, bn = c->bn, anp1 = c->anp1, bnp1 = c->bnp1, cnp1 = c->cnp1, t = c->t, tc = c->tc;
  const double dtn = c->dtn;
  const int it = c->it;
  const long long launches = c->launches;
  const bool cfl_pending = c->cfl_pending;
  auto restore = [&] {
    c->an = an; c->bn = bn; c->anp1 = anp1; c->bnp1 = bnp1; c->cnp1 = cnp1; c->t = t; c->tc = tc; c->it = it;
    c->dtn = dtn; c->launches = launches; c->cfl_pending = cfl_pending;
  };
  if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return SGPU_E_CUDA;
  }
  int r = SGPU_OK;
  for (int s = 0; s < c->prm.nst && r == SGPU_OK; ++s) {
    r = enqueue_nonlin(c);
    if (r == SGPU_OK) r = enqueue_linear(c);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  if (r != SGPU_OK || e != cudaSuccess || !graph) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    restore();
    return SGPU_E_CUDA;
  }
  bool ok = false;
  if (c->step_exec) {
    cudaGraphExecUpdateResultInfo info;
    ok = cudaGraphExecUpdate(c->step_exec, graph, &info) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      cudaGraphExecDestroy(c->step_exec);
      c->step_exec = nullptr;
    }
  }
  if (!ok) ok = cudaGraphInstantiate(&c->step_exec, graph, 0) == cudaSuccess;
  cudaGraphDestroy(graph);
  if (!ok) {
    cudaGetLastError();
    c->step_exec = nullptr;
    c->step_valid = false;
    restore();
    return SGPU_E_CUDA;
  }
  c->step_valid = true;
  c->step_key = key;
  c->step_dt = dtn;
  c->step_launches = c->launches - launches;
  return SGPU_OK;
}

// Host side of one replayed step: what enqueue_nonlin / enqueue_linear do to
// the bookkeeping, without launching.
static void replay_host(sgpu_ctx* c) {
  for (int s = 0; s < c->prm.nst; ++s) {
    c->tc = c->t + c->cnp1;
    rk_advance(c);
    it_advance(c);
  }
  if (c->step_key & 15u) c->cfl_pending = true;
  c->launches += c->step_launches;
}

extern "C" int sgpu_step_rk(sgpu_ctx* c, int nsub) {
  if (!c || nsub < 0) return SGPU_E_PARAM;
  c->press_valid = false;
  if (!c->have_state) return SGPU_E_STATE;
  // a shard needs the block exchanges between its two steps (host-driven)
  if (sharded(c)) return SGPU_E_STATE;
  const int nst = c->prm.nst;
  int s = 0;
  while (s < nsub) {
    // whole steps with an unchanged launch pattern and time step replay one
    // CUDA graph; the rest (first steps, profiling, partial steps, a step
    // whose time step changes) launch directly
    const unsigned key = (c->graphs && !c->prof && nsub - s >= nst) ? step_pattern(c) : 0xffffffffu;
    if (key != 0xffffffffu) {
      if (c->step_valid && c->step_key == key && c->step_dt == c->dtn) {
        NvtxRange nv("RK step (graph)");
        CK(cudaGraphLaunch(c->step_exec, c->stream));
        replay_host(c);
        s += nst;
        continue;
      }
      if (capture_step(c, key) == SGPU_OK) {
        CK(cudaGraphLaunch(c->step_exec, c->stream));
        s += nst;
        continue;
      }
      c->graphs = false;  // capture not possible here: launch directly from now on
    }
    // the CFL word is read back lazily (sgpu_get_scalars): no host sync per substep
    int r = enqueue_nonlin(c);
    if (r) return r;
    r = enqueue_linear(c);
    if (r) return r;
    ++s;
  }
  return SGPU_OK;
}

// The steps of sgpu_offload_steps; on an error the caller drains the copy
// streams before returning, so no copy of ur, ui is still running.
// Each slot moves in OFFLOAD_CHUNKS pieces: a piece of the next step's
// upload waits only for the same piece of this step's download, so the
// upload trails the download by one piece (1/56 of the state at eight
// pieces) instead of one slot (1/7).  At 384x193x384: 19.55 -> 20.61
// steps/s mixed, 16.39 -> 17.11 FP64 (one, eight pieces; four: 20.32, 16.84).
static int offload_enqueue(sgpu_ctx* c, double* ur, double* ui, int nsteps) {
  const Dims& g = c->g;
  const size_t n1 = (size_t)g.nyp * g.NP;  // one slot of the reference layout
  double* sre = c->stage;           // staging of the reference layout, slot k at k * n1
  double* sim = c->stage + 7 * n1;
  auto piece = [n1](int j, size_t& off, size_t& len) {
    off = n1 * j / OFFLOAD_CHUNKS;
    len = n1 * (j + 1) / OFFLOAD_CHUNKS - off;
  };
  // step 2 of a step's first substep reads slots 0-4 only (without LES): it
  // starts as soon as they are on the device and runs under the upload of
  // p_v, p_omega (slots 5, 6); the substep's step 3 waits for those.  At
  // 384x193x384: 21.1 -> 22.1 steps/s mixed, 17.5 -> 18.8 FP64 (sixteen
  // pieces per slot instead of eight: no further gain)
#ifndef SB_OFFLOAD_EARLY
#define SB_OFFLOAD_EARLY 1
#endif
  const bool early = SB_OFFLOAD_EARLY && c->iles == 0;
  for (int step = 0; step < nsteps; ++step) {
    // in: piece j of slot k waits only for the same piece of the previous
    // step to be back on the host, so it overlaps the rest of the download
    c->have_state = true;
    for (int k = 0; k < 7; ++k) {
      if (early && k == 5) {
        const int r = enqueue_nonlin(c);
        if (r) return r;
      }
      for (int j = 0; j < OFFLOAD_CHUNKS; ++j) {
        size_t off, len;
        piece(j, off, len);
        const size_t o = k * n1 + off;
        if (step > 0) CK(cudaStreamWaitEvent(c->h2d, c->down_done[k * OFFLOAD_CHUNKS + j], 0));
        CK(cudaMemcpyAsync(sre + o, ur + o, len * sizeof(double), cudaMemcpyHostToDevice, c->h2d));
        CK(cudaMemcpyAsync(sim + o, ui + o, len * sizeof(double), cudaMemcpyHostToDevice, c->h2d));
      }
      CK(cudaEventRecord(c->up_done[k], c->h2d));
      CK(cudaStreamWaitEvent(c->stream, c->up_done[k], 0));
      if (c->mixed)
        k_from_ref_mixed<<<592, 256, 0, c->stream>>>(sre + k * n1, sim + k * n1, c->st, c->stf, g, 1, k);
      else
        k_from_ref<<<592, 256, 0, c->stream>>>(sre + k * n1, sim + k * n1, c->st, g, 1, k);
      c->launches++;
    }
    int r = early ? enqueue_linear(c) : SGPU_OK;
    if (r) return r;
    r = sgpu_step_rk(c, early ? c->prm.nst - 1 : c->prm.nst);
    if (r) return r;
    // out: slot by slot, each copy as soon as its conversion is done
    for (int k = 0; k < 7; ++k) {
      if (c->mixed)
        k_to_ref_mixed<<<592, 256, 0, c->stream>>>(c->st, c->stf, sre + k * n1, sim + k * n1, g, 1, k);
      else
        k_to_ref<<<592, 256, 0, c->stream>>>(c->st, sre + k * n1, sim + k * n1, g, 1, k);
      c->launches++;
      CK(cudaEventRecord(c->out_ready[k], c->stream));
      CK(cudaStreamWaitEvent(c->d2h, c->out_ready[k], 0));
      for (int j = 0; j < OFFLOAD_CHUNKS; ++j) {
        size_t off, len;
        piece(j, off, len);
        const size_t o = k * n1 + off;
        CK(cudaMemcpyAsync(ur + o, sre + o, len * sizeof(double), cudaMemcpyDeviceToHost, c->d2h));
        CK(cudaMemcpyAsync(ui + o, sim + o, len * sizeof(double), cudaMemcpyDeviceToHost, c->d2h));
        CK(cudaEventRecord(c->down_done[k * OFFLOAD_CHUNKS + j], c->d2h));
      }
    }
  }
  CK(cudaGetLastError());
  return SGPU_OK;
}

extern "C" int sgpu_offload_steps(sgpu_ctx* c, double* ur, double* ui, int nsteps) {
  if (c) c->press_valid = false;  // the state changes
  NvtxRange nv("offload steps");
  if (!c || !ur || !ui || nsteps < 0) return SGPU_E_PARAM;
  if (sharded(c)) return SGPU_E_STATE;
  if (!c->h2d) {
    CK(cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking));
    for (int k = 0; k < 7; ++k) {
      CK(cudaEventCreateWithFlags(&c->up_done[k], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&c->out_ready[k], cudaEventDisableTiming));
    }
    for (auto& e : c->down_done) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const int r = offload_enqueue(c, ur, ui, nsteps);
  // returns only when no copy of the caller's arrays is in flight, on success
  // and on every error path
  const cudaError_t e1 = cudaStreamSynchronize(c->h2d);
  const cudaError_t e2 = cudaStreamSynchronize(c->stream);
  const cudaError_t e3 = cudaStreamSynchronize(c->d2h);
  if (r) return r;
  CK(e1);
  CK(e2);
  CK(e3);
  return SGPU_OK;
}

extern "C" int sgpu_get_scalars(sgpu_ctx* c, double* out, int n) {
  if (!c || !out) return SGPU_E_PARAM;
  int r = collect_cfl(c);
  double sc[4];
  int tc_err = 0, mlp_err = 0;
  CK(cudaMemcpyAsync(sc, c->scal, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
  if (c->chb_err) CK(cudaMemcpyAsync(&tc_err, c->chb_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  if (c->mlp_err) CK(cudaMemcpyAsync(&mlp_err, c->mlp_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const double v[12] = {sc[0], sc[1], c->t, c->cfl, c->an, c->bn, c->anp1, c->bnp1, c->cnp1, (double)c->it, c->tc, c->dtn};
  for (int i = 0; i < n && i < 12; ++i) out[i] = v[i];
  if (tc_err || mlp_err) {
    // reported once: the words are cleared, so a context whose state the
    // host restores (upload, prhs) steps on normally
    fprintf(stderr, "simson_b200: %s: a bounded wait ran out; the substep's result is not valid\n",
            tc_err ? "tensor-core Chebyshev transform" : "learned SGS model");
    if (c->chb_err) CK(cudaMemsetAsync(c->chb_err, 0, sizeof(int), c->stream));
    if (c->mlp_err) CK(cudaMemsetAsync(c->mlp_err, 0, sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SGPU_E_TIMEOUT;
  }
  // a non-finite value anywhere in u, v, w reaches the kx = kz = 0 mode of H
  // through the forward transforms within one substep, and with it px
  // (constant flux) or the mass flux
  if (r == SGPU_OK && c->have_state && !(std::isfinite(sc[0]) && std::isfinite(sc[1]))) return SGPU_E_NAN;
  return r;
}

extern "C" int sgpu_set_pencil_kernel(sgpu_ctx* c, int warp) {
  if (c) c->step_valid = false;  // the captured step launches the other kernel
  if (!c || warp < 0 || warp > 2) return SGPU_E_PARAM;
  const bool fits = pencil_warp_rows(c->g.nyp) > 0;
  if (warp == 1 && !fits) return SGPU_E_PARAM;
  c->pencil_warp = warp == 2 ? (fits && c->g.NP <= kPencilWarpMaxPencils) : warp == 1;
  return SGPU_OK;
}

extern "C" int sgpu_set_wait_limit(sgpu_ctx* c, int limit, int test_timeout) {
  if (c) c->step_valid = false;  // the limits are kernel arguments of the captured step
  if (!c || limit < 0 || test_timeout < 0 || test_timeout > 1) return SGPU_E_PARAM;
  c->wait_limit = limit;
  c->test_timeout = test_timeout;
  return SGPU_OK;
}

extern "C" int sgpu_event_record(sgpu_ctx* c, int slot_) {
  if (!c || slot_ < 0 || slot_ >= 16) return SGPU_E_PARAM;
  CK(cudaEventRecord(c->ev[slot_], c->stream));
  return SGPU_OK;
}

extern "C" int sgpu_event_elapsed(sgpu_ctx* c, int a, int b, float* ms) {
  if (!c || !ms || a < 0 || b < 0 || a >= 16 || b >= 16) return SGPU_E_PARAM;
  CK(cudaEventSynchronize(c->ev[b]));
  CK(cudaEventElapsedTime(ms, c->ev[a], c->ev[b]));
  return SGPU_OK;
}

extern "C" int sgpu_sync(sgpu_ctx* c) {
  if (!c) return SGPU_E_PARAM;
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

extern "C" long long sgpu_launch_count(sgpu_ctx* c) { return c ? c->launches : -1; }

extern "C" int sgpu_host_alloc(unsigned long long bytes, void** ptr) {
  if (!ptr) return SGPU_E_PARAM;
  *ptr = nullptr;
  CK(cudaHostAlloc(ptr, (size_t)bytes, cudaHostAllocDefault));
  return SGPU_OK;
}

extern "C" int sgpu_host_free(void* ptr) {
  if (ptr) CK(cudaFreeHost(ptr));
  return SGPU_OK;
}

// Per-kernel timing: when enabled, an event is recorded before every launch
// and the time to the next event is attributed to that kernel.
extern "C" int sgpu_profile(sgpu_ctx* c, int enable) {
  if (!c) return SGPU_E_PARAM;
  if (enable && c->pev.empty()) {
    c->pev.resize(8192);
    c->pid.resize(8192);
    for (auto& e : c->pev) CK(cudaEventCreate(&e));
  }
  c->prof = enable != 0;
  c->pnext = 0;
  return SGPU_OK;
}

extern "C" int sgpu_profile_read(sgpu_ctx* c, double* ms, int* count, int n) {
  if (!c || !ms || !count) return SGPU_E_PARAM;
  CK(cudaStreamSynchronize(c->stream));
  for (int i = 0; i < n; ++i) { ms[i] = 0.0; count[i] = 0; }
  for (int i = 0; i + 1 < c->pnext; ++i) {
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, c->pev[i], c->pev[i + 1]));
    const int id = c->pid[i];
    if (id < n) { ms[id] += t; count[id] += 1; }
  }
  c->pnext = 0;
  return SGPU_OK;
}

// Plane statistics and the amp.stat row (bla/boxamp.f; bla/wampbl.f:124-278
// for the channel, dstar = 1, one process).  The per-plane sums run on the
// device; the y-integrals of the row run here with the Clenshaw-Curtis weights
// of bla/preprbl.f:78-87 and gridy = 1 + eta (:56-58).
// xy statistics (bla/boxxys.f via bla/bla.f:2069-2107), see xys.cuh.
static int xys_setup(sgpu_ctx* c) {
  if (c->xys) return SGPU_OK;
  const Dims& g = c->g;
  constexpr int KB = 4;
  const size_t sz = 2 * (size_t)g.nz * KB * sizeof(double2);
  const size_t sx = 2 * (size_t)g.nx * XYS_NC * sizeof(double2);
  if (g.nx > 512 || sz > 227 * 1024 || sx > 227 * 1024) return SGPU_E_PARAM;
  int rc;
  if (!c->xys_twz.d && (rc = make_tw(c->xys_twz, g.nz))) return rc;
  if (!c->xys_twx.d && (rc = make_tw(c->xys_twx, g.nx))) return rc;
  const size_t plane = (size_t)g.nyp * g.nx;
  // c->xys last: its presence marks the set-up as complete
  if ((!c->xys_spec && cudaMalloc(&c->xys_spec, XYS_NF * (size_t)g.nyp * g.NP * sizeof(double2)) != cudaSuccess) ||
      (!c->xys_part &&
       cudaMalloc(&c->xys_part, (size_t)XYS_GROUPS * XYS_NACC_P * plane * sizeof(double)) != cudaSuccess) ||
      (!c->xys_u && cudaMalloc(&c->xys_u, plane * g.nz * sizeof(double)) != cudaSuccess) ||
      cudaMalloc(&c->xys, XYS_NS * plane * sizeof(double)) != cudaSuccess)
    return SGPU_E_CUDA;
  CK(cudaMemsetAsync(c->xys, 0, XYS_NS * plane * sizeof(double), c->stream));
  c->xys_sumw = 0.0;
  cudaFuncSetAttribute(k_xys_zinv<double2, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sz);
  cudaFuncSetAttribute(k_xys_zinv<float2, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sz);
  cudaFuncSetAttribute(k_xys_acc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx);
  cudaFuncSetAttribute(k_xys_acc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx);
  cudaFuncSetAttribute(k_xys_acc<false, 384>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx);
  cudaFuncSetAttribute(k_xys_acc<true, 384>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx);
  cudaFuncSetAttribute(k_box_sample, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx);
  return SGPU_OK;
}

// The 15 spectral fields of the statistics on the nx x nz grid, z physical.
static void xys_fields(sgpu_ctx* c, const double2* pr) {
  const Dims& g = c->g;
  const SgsGrid G = sgs_grid(c);
  constexpr int KB = 4;
  const size_t sz = 2 * (size_t)g.nz * KB * sizeof(double2);
  const dim3 gz((g.nx2 + KB - 1) / KB, g.nyp);
  if (c->mixed)
    k_xys_zinv<float2, KB><<<gz, 256, sz, c->stream>>>(c->stf, pr, c->xys_spec, G, c->xys_twz.plan, c->xys_twz.d,
                                                       c->alfa, c->beta);
  else
    k_xys_zinv<double2, KB><<<gz, 256, sz, c->stream>>>(c->st, pr, c->xys_spec, G, c->xys_twz.plan, c->xys_twz.d,
                                                        c->alfa, c->beta);
  c->launches++;
}

extern "C" int sgpu_box_filter_sample(sgpu_ctx* c, int factor, float* features, float* targets) {
  if (c && sharded(c)) return SGPU_E_STATE;  // reads the whole state
  if (!c || !features || !targets || factor < 1) return SGPU_E_PARAM;
  if (!c->have_state) return SGPU_E_STATE;
  const Dims& g = c->g;
  if (g.nx % factor || g.nz % factor) return SGPU_E_PARAM;
  int rc = xys_setup(c);
  if (rc) return rc;
  const int nxc = g.nx / factor, nzc = g.nz / factor;
  const size_t npts = (size_t)g.nyp * nzc * nxc;
  if (c->box_n < npts) {
    if (c->box_out) cudaFree(c->box_out);
    c->box_out = nullptr;
    c->box_n = 0;
    if (cudaMalloc(&c->box_out, npts * 16 * sizeof(float)) != cudaSuccess) return SGPU_E_CUDA;
    c->box_n = npts;
  }
  xys_fields(c, nullptr);
  const size_t sx = 2 * (size_t)g.nx * XYS_NC * sizeof(double2);
  const int nt = std::max(128, (nxc + 31) / 32 * 32);
  k_box_sample<<<dim3(nzc, g.nyp), nt, sx, c->stream>>>(c->xys_spec, sgs_grid(c), c->xys_twx.plan, c->xys_twx.d,
                                                        factor, c->box_out, c->box_out + npts * 10);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(features, c->box_out, npts * 10 * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(targets, c->box_out + npts * 10, npts * 6 * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

extern "C" int sgpu_xys_sample(sgpu_ctx* c, double dtn) {
  NvtxRange nv("xy statistics");
  if (c && sharded(c)) return SGPU_E_STATE;  // statistics read the whole state
  if (!c || !(dtn >= 0.0)) return SGPU_E_PARAM;
  if (!c->have_state) return SGPU_E_STATE;
  int rc = xys_setup(c);
  if (rc) return rc;
  const Dims& g = c->g;
  const SgsGrid G = sgs_grid(c);
  const size_t sx = 2 * (size_t)g.nx * XYS_NC * sizeof(double2);
  // the pressure entries when the pressure of this state has been computed
  const bool pres = c->press_valid && c->press;
  xys_fields(c, pres ? c->press : nullptr);
  const int nt = (g.nx + 31) / 32 * 32;
  const dim3 gr(XYS_GROUPS, g.nyp);
  const double cw = dtn / (double)g.nz;
  // the 384-thread instances (more registers per thread) whenever nx fits
  if (pres && nt <= 384)
    k_xys_acc<true, 384><<<gr, nt, sx, c->stream>>>(c->xys_spec, c->xys_part, c->xys_u, G, c->xys_twx.plan,
                                                    c->xys_twx.d, cw);
  else if (pres)
    k_xys_acc<true><<<gr, nt, sx, c->stream>>>(c->xys_spec, c->xys_part, c->xys_u, G, c->xys_twx.plan, c->xys_twx.d,
                                               cw);
  else if (nt <= 384)
    k_xys_acc<false, 384><<<gr, nt, sx, c->stream>>>(c->xys_spec, c->xys_part, c->xys_u, G, c->xys_twx.plan,
                                                     c->xys_twx.d, cw);
  else
    k_xys_acc<false><<<gr, nt, sx, c->stream>>>(c->xys_spec, c->xys_part, c->xys_u, G, c->xys_twx.plan, c->xys_twx.d,
                                                cw);
  const size_t plane = (size_t)g.nyp * g.nx;
  const int nb = (int)((plane + 255) / 256);
  k_xys_add<<<nb, 256, 0, c->stream>>>(c->xys_part, c->xys, G, pres ? XYS_NACC_P : XYS_NACC);
  k_xys_minmax<<<nb, 256, 0, c->stream>>>(c->xys_u, c->xys, G);
  c->launches += 3;
  c->xys_sumw += dtn;
  CK(cudaGetLastError());
  return SGPU_OK;
}

extern "C" int sgpu_xys_get(sgpu_ctx* c, double* xys, double* sumw) {
  if (!c || !xys) return SGPU_E_PARAM;
  const Dims& g = c->g;
  const size_t bytes = XYS_NS * (size_t)g.nyp * g.nx * sizeof(double);
  if (!c->xys) {
    memset(xys, 0, bytes);
  } else {
    CK(cudaMemcpyAsync(xys, c->xys, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  if (sumw) *sumw = c->xys_sumw;
  return SGPU_OK;
}

extern "C" int sgpu_xys_reset(sgpu_ctx* c) {
  if (!c) return SGPU_E_PARAM;
  if (c->xys) CK(cudaMemsetAsync(c->xys, 0, XYS_NS * (size_t)c->g.nyp * c->g.nx * sizeof(double), c->stream));
  c->xys_sumw = 0.0;
  return SGPU_OK;
}

// Pressure of the current state (press.cuh; bla/nonlinp.f + bla/linearp.f as
// bla/bla.f:2486-2527 runs them); FP64 arithmetic under either storage.
extern "C" int sgpu_pressure(sgpu_ctx* c, double* pr, double* pi) {
  NvtxRange nv("pressure");
  if (c && sharded(c)) return SGPU_E_STATE;  // reads the whole state
  if (!c || !pr || !pi) return SGPU_E_PARAM;
  if (!c->have_state) return SGPU_E_STATE;
  const Dims& g = c->g;
  const int n = g.nyp;
  if (n < 9) return SGPU_E_PARAM;
  const size_t fld = (size_t)n * g.NP;
  if (!c->press) {
    // second-derivative weights at y = +1 and y = -1 on the Gauss-Lobatto
    // points (bla/preprbl.f:90-118: wd1(:,2) and wd1(:,4))
    const double pi_ = 3.1415926535897932385;
    std::vector<double> wd(2 * (size_t)n, 0.0), cw(n, 1.0);
    cw[0] = 0.5;
    cw[n - 1] = 0.5;
    double sgn = 1.0;
    for (int i = 1; i <= n; ++i) {
      sgn = -sgn;
      const double kk = (double)(i - 1) * (double)(i - 1);
      for (int y = 1; y <= n; ++y) {
        const double cs = cos(pi_ * (double)((i - 1) * (y - 1)) / (double)(n - 1));
        wd[y - 1] = wd[y - 1] + kk * (kk - 1.) / 3. * cw[y - 1] * cw[i - 1] * cs * (2. / (double)(n - 1));
        wd[n + y - 1] =
            wd[n + y - 1] - kk * (kk - 1.) / 3. * cw[y - 1] * cw[i - 1] * sgn * cs * (2. / (double)(n - 1));
      }
    }
    if (cudaMalloc(&c->press_wd, 2 * (size_t)n * sizeof(double)) != cudaSuccess) {
      c->press_wd = nullptr;
      return SGPU_E_CUDA;
    }
    if (cudaMalloc(&c->press, fld * sizeof(double2)) != cudaSuccess) {
      cudaFree(c->press_wd);
      c->press_wd = nullptr;
      c->press = nullptr;
      return SGPU_E_CUDA;
    }
    CK(cudaMemcpyAsync(c->press_wd, wd.data(), wd.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->press, 0, fld * sizeof(double2), c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  const sgpu_params& P = c->prm;
  // step-2 transforms of u, omega and the products H, 2E (nonlinp.f)
  dim3 gz((g.nx2 + c->kb - 1) / c->kb, n);
  const size_t s_z = smem_fft(g.nzp, c->kb, sizeof(double2));
  if (c->mixed)
    launch_zinv<double, sgpu_ctx::kb, float>(gz, s_z, c->stream, c->stf, c->zb, g, c->twz.plan, c->twz.d, c->alfa,
                                             c->beta, 0);
  else
    launch_zinv<double, sgpu_ctx::kb, double>(gz, s_z, c->stream, c->st, c->zb, g, c->twz.plan, c->twz.d,
                                              c->alfa, c->beta, 0);
  const size_t s_xp = 2 * (size_t)g.nxp * 3 * sizeof(double2);
  cudaFuncSetAttribute(k_xpass_p, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s_xp);
  k_xpass_p<<<dim3(g.nzp, n), 256, s_xp, c->stream>>>(c->zb, g, c->twx.plan, c->twx.d, P.rot, ctx_fringe(c));
  const size_t fz = (size_t)n * g.nzp * g.nx2;  // one field of zb
  launch_zfwd<double, sgpu_ctx::kb, double>(gz, s_z, c->stream, c->zb, czf(c, 0), g, c->twz.plan, c->twz.d,
                                            nullptr, 0.0);  // H1, H2, H3
  launch_zfwd<double, sgpu_ctx::kb, double>(gz, s_z, c->stream, c->zb + 3 * fz, czf(c, 3), g, c->twz.plan,
                                            c->twz.d, nullptr, 0.0);  // 2E (fields 4, 5 overwritten below)
  k_press_div<<<(unsigned)((fld + 255) / 256), 256, 0, c->stream>>>(czf(c, 0), g, c->alfa, c->beta);
  // Chebyshev coefficients (linearp.f:89-114)
  const double cn = 1.0 / ((double)g.nxp * (double)g.nzp);
  launch_cheb_t<double, sgpu_ctx::pb, double, double>(c, czf(c, 0), fld, czf(c, 4), fld, 2, 0, cn, 1, c->twy.d);
  launch_cheb_t<double, sgpu_ctx::pb, double, double>(c, czf(c, 3), fld, czf(c, 6), fld, 1, 0,
                                                      1.0 / (2.0 * (double)g.nxp * (double)g.nzp), 1, c->twy.d);
  PressArgs A;
  A.CD = czf(c, 4); A.CH2 = czf(c, 5); A.CE = czf(c, 6);
  A.PH2 = czf(c, 1); A.PE = czf(c, 3);
  A.V = slot(c, 1);
  A.Vf = c->mixed ? c->stf + fld : nullptr;
  A.X = czf(c, 7);
  A.Q = reinterpret_cast<double*>(czf(c, 8)); A.Cc = A.Q + fld;
  A.Dd = reinterpret_cast<double*>(czf(c, 9)); A.Ee = A.Dd + fld;
  A.wd = c->press_wd; A.alfa = c->alfa; A.beta = c->beta;
  A.re = P.re;
  A.c4t = 1. / c->dtn * (double)(1 - 1 / c->it);
  A.cn = cn;
  A.e2n = 2. * (double)g.nxp * (double)g.nzp;
  A.cim = 0;
  k_press<<<(g.NP + 127) / 128, 128, 0, c->stream>>>(A, g);
  // back to physical y (vchbb), the oddball plane left out (linearp.f:64)
  launch_cheb_t<double, sgpu_ctx::pb, double, double>(c, czf(c, 7), fld, c->press, fld, 1, 1, 1.0, 1, c->twy.d);
  c->launches += 9;
  CK(cudaGetLastError());
  k_to_ref<<<592, 256, 0, c->stream>>>(c->press, c->stage, c->stage + fld, g, 1);
  CK(cudaMemcpyAsync(pr, c->stage, fld * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(pi, c->stage + fld, fld * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->press_valid = true;
  return SGPU_OK;
}

// Training of the learned SGS model (mlp_train.cuh): iters full-batch Adam
// steps on n host samples, then the loss and the gradient at the final
// weights.  Device buffers are allocated for the call and freed after it.
extern "C" int sgpu_sgs_mlp_train(sgpu_ctx* c, float* params, float* adam_m, float* adam_v, int* adam_step,
                                  const float* x, const float* t, long long n, int iters, float lr, float* loss,
                                  float* grad) {
  NvtxRange nv("learned SGS training");
  if (!c || !params || !adam_m || !adam_v || !adam_step || !x || !t || n < 1 || iters < 0 || !(lr >= 0.0f))
    return SGPU_E_PARAM;
  const long long nchunk = (n + MLP_CHUNK - 1) / MLP_CHUNK;
  if (nchunk > 0x7fffffffLL) return SGPU_E_PARAM;
  const size_t np = MLP_NPAR, np1 = MLP_NPAR + 1;
  float *d_par = nullptr, *d_m = nullptr, *d_v = nullptr, *d_g = nullptr, *d_part = nullptr, *d_x = nullptr,
        *d_t = nullptr;
  auto release = [&] {
    for (float* q : {d_par, d_m, d_v, d_g, d_part, d_x, d_t})
      if (q) cudaFree(q);
  };
  if (cudaMalloc(&d_par, np * sizeof(float)) != cudaSuccess || cudaMalloc(&d_m, np * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&d_v, np * sizeof(float)) != cudaSuccess || cudaMalloc(&d_g, np1 * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&d_part, (size_t)nchunk * np1 * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&d_x, (size_t)n * MLP_NIN * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&d_t, (size_t)n * MLP_NOUT * sizeof(float)) != cudaSuccess) {
    release();
    return SGPU_E_CUDA;
  }
  int rc = SGPU_OK;
  auto chk = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == SGPU_OK) rc = cuda_fail(e, "sgs mlp training");
  };
  chk(cudaMemcpyAsync(d_par, params, np * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  chk(cudaMemcpyAsync(d_m, adam_m, np * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  chk(cudaMemcpyAsync(d_v, adam_v, np * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  chk(cudaMemcpyAsync(d_x, x, (size_t)n * MLP_NIN * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  chk(cudaMemcpyAsync(d_t, t, (size_t)n * MLP_NOUT * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  chk(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_TRAIN_SMEM));
  const int gb = (int)((np1 + 255) / 256);
  for (int it = 0; it <= iters && rc == SGPU_OK; ++it) {
    k_mlp_grad<<<(unsigned)nchunk, MLP_TRAIN_THREADS, MLP_TRAIN_SMEM, c->stream>>>(d_par, d_x, d_t, n, d_part);
    k_mlp_reduce<<<gb, 256, 0, c->stream>>>(d_part, (int)nchunk, d_g);
    c->launches += 2;
    if (it == iters) break;  // the gradient and loss at the final weights
    const int step = ++*adam_step;
    const float c1 = (float)(1.0 / (1.0 - pow(0.9, (double)step)));
    const float c2 = (float)(1.0 / (1.0 - pow(0.999, (double)step)));
    k_mlp_adam<<<gb, 256, 0, c->stream>>>(d_par, d_m, d_v, d_g, lr, c1, c2);
    c->launches++;
    chk(cudaGetLastError());
  }
  chk(cudaGetLastError());
  float sse = 0.0f;
  chk(cudaMemcpyAsync(params, d_par, np * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  chk(cudaMemcpyAsync(adam_m, d_m, np * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  chk(cudaMemcpyAsync(adam_v, d_v, np * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  if (grad) chk(cudaMemcpyAsync(grad, d_g, np * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  chk(cudaMemcpyAsync(&sse, d_g + np, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  chk(cudaStreamSynchronize(c->stream));
  if (loss) *loss = sse / (6.0f * (float)n);
  release();
  return rc;
}

extern "C" int sgpu_amplitudes(sgpu_ctx* c, double* amp, double* row) {
  if (c && sharded(c)) return SGPU_E_STATE;  // statistics read the whole state
  if (!c || !amp) return SGPU_E_PARAM;
  if (!c->have_state) return SGPU_E_STATE;
  const Dims& g = c->g;
  if (c->mixed)
    k_amp<float><<<g.nyp, 256, 0, c->stream>>>(c->stf, g, c->alfa, c->beta, c->ampd);
  else
    k_amp<double><<<g.nyp, 256, 0, c->stream>>>(c->st, g, c->alfa, c->beta, c->ampd);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(amp, c->ampd, 20 * (size_t)g.nyp * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  double sc[4];
  CK(cudaMemcpyAsync(sc, c->scal, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (!row) return SGPU_OK;
  const int n = g.nyp;
  const double pi = 3.1415926535897932385;
  std::vector<double> wint(n), gridy(n), a(20 * (size_t)n);
  for (int y = 0; y < n; ++y) {
    double wv = -.5;
    for (int i = 1; i <= (n + 1) / 2 - 2; ++i)
      wv = wv + cos(pi * (double)(2 * i * y) / (double)(n - 1)) / (double)((2 * i) * (2 * i) - 1);
    wv = wv + .5 * cos(pi * (double)y) / (double)((n - 1) * (n - 1) - 1);
    wv = -4. / (double)(n - 1) * wv;
    if (y == 0 || y == n - 1) wv = wv * .5;
    wint[y] = wv;
    gridy[y] = 1. + cos(pi * (double)y / (double)(n - 1));
  }
  memcpy(a.data(), amp, a.size() * sizeof(double));
  auto A = [&](int y, int k) -> double& { return a[(size_t)(k - 1) * n + y]; };  // amp(y+1, k)
  double sum[21] = {0};
  for (int y = 0; y < n; ++y) {
    A(y, 8) = -A(y, 8);
    A(y, 13) = A(y, 9);
  }
  for (int i = 1; i <= 10; ++i)
    for (int y = 0; y < n; ++y) sum[i] += A(y, i) * wint[y];
  for (int y = 0; y < n; ++y) sum[13] += A(y, 13) * wint[y];
  double delta[4] = {0, 0, 0, 0};
  for (int y = 0; y < n; ++y) {
    if (delta[1] == 0. && A(y, 13) <= 0.99) {
      if (A(y, 13) == 0.99 || y == 0)
        delta[1] = gridy[y];
      else
        delta[1] = gridy[y] + (0.99 - A(y, 13)) * (gridy[y - 1] - gridy[y]) / (A(y - 1, 13) - A(y, 13));
    }
    delta[2] += (1. - A(y, 13)) * wint[y];
    delta[3] += A(y, 13) * (1. - A(y, 13)) * wint[y];
  }
  for (int j = 1; j <= 7; ++j) sum[j] = sqrt(sum[j] * .5);
  const double wb = sum[10] * .5;
  const double e0 = sqrt((sum[9] + sum[10]) * .5);
  const double tau1 = A(0, 12), tau2 = A(n - 1, 12);
  const double hplus = sqrt((fabs(tau1) + fabs(tau2)) * c->prm.re / 2.);
  const double r[19] = {c->t, sum[1], sum[2], sum[3], sum[4], sum[5], sum[6], sum[7], sum[8], e0, hplus, sc[0],
                        sum[13] * c->prm.re / 2., tau1, tau2, delta[1], delta[2], delta[3], wb};
  memcpy(row, r, sizeof(r));
  return SGPU_OK;
}

// Buffers, transforms and Delta^2 of the eddy-viscosity and learned models.
// les_gu with at least n fields (zeroed when (re)allocated)
static int les_gu_ensure(sgpu_ctx* c, int n) {
  if (c->les_gu_n >= n) return SGPU_OK;
  const size_t fld = (size_t)c->g.nyp * c->g.NP;
  if (c->les_gu) cudaFree(c->les_gu);
  c->les_gu_n = 0;
  if (cudaMalloc(&c->les_gu, n * fld * sizeof(double2)) != cudaSuccess) {
    c->les_gu = nullptr;
    return SGPU_E_CUDA;
  }
  CK(cudaMemsetAsync(c->les_gu, 0, n * fld * sizeof(double2), c->stream));
  c->les_gu_n = n;
  return SGPU_OK;
}

static int sgs_setup(sgpu_ctx* c) {
  const Dims& g = c->g;
  const size_t fld = (size_t)g.nyp * g.NP;
  if (g.nx % 4 || g.nz % 4) return SGPU_E_PARAM;
  constexpr int KB = 4;
  const size_t sz = 2 * (size_t)g.nz * KB * sizeof(double2);
  const size_t sx11 = 2 * (size_t)g.nx * 11 * sizeof(double2);
  if (sz > 227 * 1024 || sx11 > 227 * 1024) return SGPU_E_PARAM;
  if (!c->sgs.spec9) {
    int rc;
    if ((rc = make_tw(c->sgs_twz, g.nz)) || (rc = make_tw(c->sgs_twx, g.nx))) return rc;
    const size_t pl = (size_t)g.nyp * g.nz * g.nx;  // one real field on the nx x nz grid
    if (cudaMalloc(&c->sgs.spec9, 9 * fld * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&c->sgs.phys10, 10 * pl * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->sgs.filt21, 21 * (size_t)g.nyp * g.nz * (g.nx / 4) * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&c->sgs.numden, 2 * pl * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->sgs.cxy, (size_t)g.nyp * g.nx * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->sgs.tauz6, 6 * fld * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&c->sgs.tau, 6 * fld * sizeof(double2)) != cudaSuccess ||
        cudaMalloc(&c->sgs_delta2, (size_t)g.nyp * sizeof(double)) != cudaSuccess)
      return SGPU_E_CUDA;
    int rg = les_gu_ensure(c, 3);
    if (rg) return rg;
    const int sm[4] = {(int)sz, (int)sx11, (int)(2 * (size_t)g.nx * 3 * sizeof(double2)),
                       (int)(2 * (size_t)g.nx * 5 * sizeof(double2))};
    cudaFuncSetAttribute(k_sgs_zinv<double2, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm[0]);
    cudaFuncSetAttribute(k_sgs_zinv<float2, KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm[0]);
    cudaFuncSetAttribute(k_sgs_zfilt<KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm[0]);
    cudaFuncSetAttribute(k_sgs_zfwd<KB>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm[0]);
    cudaFuncSetAttribute(k_sgs_xpass1, cudaFuncAttributeMaxDynamicSharedMemorySize, sm[1]);
    cudaFuncSetAttribute(k_sgs_xpass2, cudaFuncAttributeMaxDynamicSharedMemorySize, sm[1]);
    cudaFuncSetAttribute(k_sgs_tau_x, cudaFuncAttributeMaxDynamicSharedMemorySize, sm[2]);
    cudaFuncSetAttribute(k_sgs_xinv9, cudaFuncAttributeMaxDynamicSharedMemorySize, sm[3]);
  }
  // Delta^2 = (dx dz dy)^(2/3), dy the geometric mean of the two
  // neighbouring Gauss-Lobatto spacings, 1 - eta_2 at the walls
  const double pi = 3.1415926535897932385;
  std::vector<double> eta(g.nyp), d2(g.nyp);
  for (int y = 0; y < g.nyp; ++y) eta[y] = cos(pi * (double)y / (double)(g.nyp - 1));
  for (int y = 0; y < g.nyp; ++y) {
    const double dy = (y == 0 || y == g.nyp - 1) ? 1. - eta[1] : sqrt((eta[y + 1] - eta[y]) * (eta[y] - eta[y - 1]));
    d2[y] = pow(c->prm.xl / (double)g.nx * c->prm.zl / (double)g.nz * dy, 2. / 3.);
  }
  CK(cudaMemcpyAsync(c->sgs_delta2, d2.data(), g.nyp * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

// ADM-RT large-eddy model (bla/rparamles.f, bla/bla.f:1489-1518, 2212-2231):
// filter tables on the host (les_filter.h), gu and the tables on the device.
// ---------------------------------------------------------------------------
// Spatial simulation: fringe forcing towards a base flow (bla/fring.f,
// bla/ffun.f; the base flow of bla/bflow.f is computed by the caller)
// ---------------------------------------------------------------------------
// Smooth step of bla/step.f: 0 up to 0.02, 1 above 0.98,
// 1 / (1 + exp(1/(x - 1) + 1/x)) between.
static double fringe_step(double x) {
  if (x <= 0.02) return 0.0;
  if (x <= 0.98) return 1.0 / (1.0 + exp(1.0 / (x - 1.0) + 1.0 / x));
  return 1.0;
}

// The fringe function of bla/ffun.f at the nxp physical x points (x pair k of
// the reference, fring1(k) / fring2(k), is points 2k-2 and 2k-1 here): fmax
// (S((x - fstart)/frise) - S((x - fend)/ffall + 1)) over the x range the
// reference fills (the fringe start and end mapped into the box around xsc;
// a fringe across the box end is filled in two parts with fmax added), zero
// elsewhere.
extern "C" int sgpu_fringe_function(const sgpu_fringe* f, int nxp, double xl, double* lam) {
  if (!f || !lam || nxp < 2 || (nxp & 1) || !(xl > 0.0) || !(f->frise > 0.0) || !(f->ffall > 0.0))
    return SGPU_E_PARAM;
  for (int j = 0; j < nxp; ++j) lam[j] = 0.0;
  const double r = 0.499999999999999999;  // rounding offset of the int() below, as bla/ffun.f declares it
  const double dnx = xl / (double)nxp;
  const double fstc = f->fstart + (double)(long long)((f->xsc - f->fstart) / xl + r) * xl;
  const double fenc = f->fend + (double)(long long)((f->xsc - f->fend) / xl + r) * xl;
  const int nh = nxp / 2;
  const int xstart = (int)((double)nh * (fstc - f->xsc + xl / 2.0) / xl) + 1;
  const int xend = (int)((double)nh * (fenc - f->xsc + xl / 2.0) / xl) + 1;
  const bool wrap = xstart > xend;  // the fringe crosses the box end: two ranges
  for (int i = wrap ? 0 : 1; i <= 1; ++i) {
    const int xst = (i == 0) ? 1 : xstart;
    const int xen = std::max(xend, (i == 0) ? 1 : (wrap ? nh : 1));
    if (xst < 1 || xen > nh) return SGPU_E_PARAM;  // outside the box: the reference would index past fring1
    for (int x = xst; x <= xen; ++x) {
      const double xc1 = (double)(2 * x - 1 - nh - 1) * dnx + f->xsc;
      double f1 = f->fmax * (fringe_step((xc1 - fstc) / f->frise) - fringe_step((xc1 - fenc) / f->ffall + 1.0));
      const double xc2 = xc1 + dnx;
      double f2 = f->fmax * (fringe_step((xc2 - fstc) / f->frise) - fringe_step((xc2 - fenc) / f->ffall + 1.0));
      if (wrap) {
        f1 = f1 + f->fmax;
        f2 = f2 + f->fmax;
      }
      lam[2 * (x - 1)] = f1;
      lam[2 * (x - 1) + 1] = f2;
    }
  }
  return SGPU_OK;
}

static int fringe_alloc(sgpu_ctx* c) {
  const Dims& g = c->g;
  const size_t nb = 3 * (size_t)g.nyp * g.nxp;
  if (!c->fr_lam && cudaMalloc(&c->fr_lam, (size_t)g.nxp * sizeof(double)) != cudaSuccess) {
    c->fr_lam = nullptr;
    return SGPU_E_CUDA;
  }
  if (!c->fr_base) {
    if (cudaMalloc(&c->fr_base, nb * sizeof(double)) != cudaSuccess) {
      c->fr_base = nullptr;
      return SGPU_E_CUDA;
    }
    CK(cudaMemsetAsync(c->fr_base, 0, nb * sizeof(double), c->stream));
  }
  return SGPU_OK;
}

extern "C" int sgpu_set_fringe(sgpu_ctx* c, const sgpu_fringe* f) {
  if (!c) return SGPU_E_PARAM;
  c->step_valid = false;   // the captured step no longer matches
  c->press_valid = false;  // the pressure includes the fringe force
  if (!f || f->fmax == 0.0) {
    c->fringe = false;
    return SGPU_OK;
  }
  if (!(f->fmax > 0.0)) return SGPU_E_PARAM;
  const Dims& g = c->g;
  std::vector<double> lam((size_t)g.nxp);
  int r = sgpu_fringe_function(f, g.nxp, c->prm.xl, lam.data());
  if (r) return r;
  r = fringe_alloc(c);
  if (r) return r;
  CK(cudaMemcpyAsync(c->fr_lam, lam.data(), lam.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->fringe = true;
  return SGPU_OK;
}

// bu1, bu2(nxp/2+1, nyp, 3) of the reference (bla/bflow.f): the base flow
// u, v, w in physical space at the even (bu1) and odd (bu2) x points.
extern "C" int sgpu_set_base_flow(sgpu_ctx* c, const double* bu1, const double* bu2) {
  if (!c || (bu1 == nullptr) != (bu2 == nullptr)) return SGPU_E_PARAM;
  c->press_valid = false;
  const Dims& g = c->g;
  int r = fringe_alloc(c);
  if (r) return r;
  const size_t nb = 3 * (size_t)g.nyp * g.nxp;
  if (!bu1) {
    CK(cudaMemsetAsync(c->fr_base, 0, nb * sizeof(double), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return SGPU_OK;
  }
  const int nh = g.nxp / 2, ld = nh + 1;  // leading dimension nxp/2+1
  std::vector<double> b(nb);
  for (int i = 0; i < 3; ++i)
    for (int y = 0; y < g.nyp; ++y)
      for (int x = 0; x < nh; ++x) {
        const size_t src = (size_t)x + (size_t)ld * ((size_t)y + (size_t)g.nyp * i);
        double* row = b.data() + ((size_t)i * g.nyp + y) * g.nxp;
        row[2 * x] = bu1[src];
        row[2 * x + 1] = bu2[src];
      }
  CK(cudaMemcpyAsync(c->fr_base, b.data(), nb * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

extern "C" int sgpu_set_les(sgpu_ctx* c, const sgpu_les_params* p) {
  if (c) c->step_valid = false;  // the captured step no longer matches
  if (c && sharded(c) && p && p->iles != 0) return SGPU_E_PARAM;  // LES needs the whole domain
  if (!c || !p) return SGPU_E_PARAM;
  if (p->iles == 0) {
    c->iles = 0;
    return SGPU_OK;
  }
  const Dims& g = c->g;
  if (p->iles == 2) {
    // eddy viscosity: cs = 0 dynamic (Germano/Lilly), else fixed C = cs^2
    if (p->ineg < 0 || p->ineg > 2 || (p->cs != 0.0 && p->ineg != 1) || !(p->cs >= 0.0)) return SGPU_E_PARAM;
    int rc = sgs_setup(c);
    if (rc) return rc;
    c->les_cs = p->cs;
    c->les_ineg = p->ineg;
    c->iles = 2;
    return SGPU_OK;
  }
  if (p->iles != 1 && p->iles != 3) {
    fprintf(stderr, "simson_b200: sgpu_set_les: iles=%d not supported (0, 1, 2 or 3)\n", p->iles);
    return SGPU_E_PARAM;
  }
  if (p->iles == 3 && (p->ineg < 0 || p->ineg > 2 || (p->cs != 0.0 && p->ineg != 1) || !(p->cs >= 0.0)))
    return SGPU_E_PARAM;
  if (!(p->cutoff_inv >= 1.0) || p->iord < 0 || p->iord > 5 || p->ihighorder < 0 || p->ihighorder > 2 ||
      !(p->chi >= 0.0))
    return SGPU_E_PARAM;
  if (g.nyp < 7) return SGPU_E_PARAM;
  LesFilter F;
  if (!les_filter_build(g.nyp, g.nx, g.nz, 1.0 / p->cutoff_inv, p->iord, F)) return SGPU_E_PARAM;
  std::vector<double> rows;
  les_filter_rows(F, rows);
  if (!c->les_coef) {
    if (cudaMalloc(&c->les_coef, rows.size() * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->les_lpf, (size_t)g.NP * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->les_filt, (size_t)g.NP * sizeof(double)) != cudaSuccess)
      return SGPU_E_CUDA;
  }
  {
    // ADM-RT filters u, v, w; the HPF model also omega_x, omega_z
    // (bla/linearbl.f:1965-2060), from which it forms the filtered gradients
    const int rg = les_gu_ensure(c, p->iles == 3 ? 5 : 3);
    if (rg) return rg;
  }
  if (p->iles == 3) {
    const int rs = sgs_setup(c);
    if (rs) return rs;
    c->les_cs = p->cs;
    c->les_ineg = p->ineg;
    c->hpf_dyn = (p->cs == 0.0);
    if (c->hpf_dyn) {
      // the secondary filter of the dynamic procedure (bla/bla.f:1520-1545)
      LesFilter F2;
      if (!les_filter_build(g.nyp, g.nx, g.nz, 1.0 / p->cutoff_inv, p->iord, F2, true)) return SGPU_E_PARAM;
      const size_t fld = (size_t)g.nyp * g.NP;
      const size_t pl = (size_t)g.nyp * g.nz * g.nx;
      if (!c->les_lpf2) {
        if (cudaMalloc(&c->les_lpf2, (size_t)g.NP * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&c->les_filt2, (size_t)g.NP * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&c->les_gu2, 5 * fld * sizeof(double2)) != cudaSuccess ||
            cudaMalloc(&c->hpf_s2, 6 * pl * sizeof(double)) != cudaSuccess)
          return SGPU_E_CUDA;
        CK(cudaMemsetAsync(c->les_gu2, 0, 5 * fld * sizeof(double2), c->stream));
      }
      CK(cudaMemcpyAsync(c->les_lpf2, F2.lpfxz.data(), (size_t)g.NP * sizeof(double), cudaMemcpyHostToDevice,
                         c->stream));
      CK(cudaMemcpyAsync(c->les_filt2, F2.filtxz.data(), (size_t)g.NP * sizeof(double), cudaMemcpyHostToDevice,
                         c->stream));
      CK(cudaStreamSynchronize(c->stream));
    }
  }
  CK(cudaMemcpyAsync(c->les_coef, rows.data(), rows.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->les_lpf, F.lpfxz.data(), (size_t)g.NP * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->les_filt, F.filtxz.data(), (size_t)g.NP * sizeof(double), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->les_fact2 = F.fact2;
  c->les_factm2 = F.factm2;
  c->les_mode = p->ihighorder;
  c->les_iord = p->iord;
  c->les_chi = p->chi;  // chi_scaled = chi / dstar, dstar = 1
  c->iles = p->iles;
  return SGPU_OK;
}

// gur, gui(memnx, memny, memnz, 1..3) of the reference: the high-pass
// filtered velocities the next step 2 relaxes towards zero.
extern "C" int sgpu_download_les(sgpu_ctx* c, double* gr, double* gi) {
  if (!c || !gr || !gi) return SGPU_E_PARAM;
  if (c->iles < 1) return SGPU_E_STATE;
  const size_t n = 3 * (size_t)c->g.nyp * c->g.NP;
  k_to_ref<<<592, 256, 0, c->stream>>>(c->les_gu, c->stage, c->stage + n, c->g, 3);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(gr, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(gi, c->stage + n, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

// tau_ij of the last eddy-viscosity evaluation (taur, taui slots 1..6:
// 11 12 13 22 23 33) in the reference layout.
extern "C" int sgpu_download_sgs_stress(sgpu_ctx* c, double* tr, double* ti) {
  if (!c || !tr || !ti) return SGPU_E_PARAM;
  if (c->iles < 2) return SGPU_E_STATE;
  const size_t n = 6 * (size_t)c->g.nyp * c->g.NP;  // the staging area holds 7 slots
  k_to_ref<<<592, 256, 0, c->stream>>>(c->sgs.tau, c->stage, c->stage + n, c->g, 6);
  c->launches++;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(tr, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(ti, c->stage + n, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

// Learned SGS model (no counterpart in the reference): weights and scalings,
// then every substep uses it in place of the eddy-viscosity stress.
static int mlp_image_upload(sgpu_ctx* c, const sgpu_sgs_mlp* p) {
  if (!p->w1 || !p->b1 || !p->w2 || !p->b2 || !p->w3 || !p->b3) return SGPU_E_PARAM;
  std::vector<unsigned char> img(MLP_IMAGE_BYTES);
  mlp_build_image(p->w1, p->b1, p->w2, p->b2, p->w3, p->b3, img.data());
  if (!c->mlp_image) {
    if (cudaMalloc(&c->mlp_image, MLP_IMAGE_BYTES) != cudaSuccess ||
        cudaMalloc(&c->mlp_err, sizeof(int)) != cudaSuccess)
      return SGPU_E_CUDA;
    cudaFuncSetAttribute(k_sgs_mlp, cudaFuncAttributeMaxDynamicSharedMemorySize, MLP_SMEM_LAUNCH);
  }
  CK(cudaMemcpyAsync(c->mlp_image, img.data(), MLP_IMAGE_BYTES, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->mlp_err, 0, sizeof(int), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->mlp_s_in = p->s_in;
  c->mlp_s_y = p->s_y;
  c->mlp_s_out = p->s_out;
  return SGPU_OK;
}

extern "C" int sgpu_set_sgs_mlp(sgpu_ctx* c, const sgpu_sgs_mlp* p) {
  if (c) c->step_valid = false;  // the captured step no longer matches
  if (!c || !p) return SGPU_E_PARAM;
  int rc = mlp_image_upload(c, p);
  if (rc) return rc;
  if ((rc = sgs_setup(c))) return rc;
  if (!c->mlp_tau && cudaMalloc(&c->mlp_tau, 6 * (size_t)c->g.nyp * c->g.nz * c->g.nx * sizeof(double)) != cudaSuccess)
    return SGPU_E_CUDA;
  c->iles = 4;
  return SGPU_OK;
}

// Per-plane fallback of the learned model (no counterpart in the reference):
// planes whose predicted backscatter exceeds the bound take the eddy-viscosity
// stress of bla/les.f (dynamic when cs = 0, clipping ineg) for that substep.
extern "C" int sgpu_set_sgs_fallback(sgpu_ctx* c, int enable, double bound, double cs, int ineg) {
  if (c) c->step_valid = false;  // the captured step no longer matches
  if (!c) return SGPU_E_PARAM;
  if (!enable) {
    c->sgs_fb = false;
    return SGPU_OK;
  }
  if (!(bound == bound) || ineg < 0 || ineg > 2 || !(cs >= 0.0) || (cs != 0.0 && ineg != 1)) return SGPU_E_PARAM;
  int rc = sgs_setup(c);
  if (rc) return rc;
  const int n = c->g.nyp;
  if (!c->sgs_flags) {
    if (cudaMalloc(&c->sgs_flags, n * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&c->sgs_bsums, 2 * (size_t)n * sizeof(double)) != cudaSuccess)
      return SGPU_E_CUDA;
    CK(cudaMemsetAsync(c->sgs_flags, 0, n * sizeof(int), c->stream));
    CK(cudaMemsetAsync(c->sgs_bsums, 0, 2 * (size_t)n * sizeof(double), c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  c->sgs_fb = true;
  c->sgs_fb_bound = bound;
  c->les_cs = cs;
  c->les_ineg = ineg;
  return SGPU_OK;
}

extern "C" int sgpu_sgs_fallback_planes(sgpu_ctx* c, int* planes, double* sums) {
  if (!c || !planes) return SGPU_E_PARAM;
  if (!c->sgs_flags) return SGPU_E_STATE;
  const int n = c->g.nyp;
  CK(cudaMemcpyAsync(planes, c->sgs_flags, n * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  if (sums) CK(cudaMemcpyAsync(sums, c->sgs_bsums, 2 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return SGPU_OK;
}

// The MLP alone on n host feature rows x[n][10] -> y[n][6] (the kernel the
// step uses, features given instead of formed from the velocity gradient).
extern "C" int sgpu_sgs_mlp_eval(sgpu_ctx* c, const sgpu_sgs_mlp* p, const float* x, float* y, long long n) {
  if (!c || !p || !x || !y || n < 0) return SGPU_E_PARAM;
  if (n == 0) return SGPU_OK;
  int rc = mlp_image_upload(c, p);
  if (rc) return rc;
  float *dx = nullptr, *dy = nullptr;
  if (cudaMalloc(&dx, (size_t)n * MLP_IN * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&dy, (size_t)n * MLP_OUT * sizeof(float)) != cudaSuccess) {
    cudaFree(dx);
    return SGPU_E_CUDA;
  }
  MlpArgs A{};
  A.image = c->mlp_image;
  A.mode = 0;
  A.n = n;
  A.x = dx;
  A.y = dy;
  A.s_in = p->s_in;
  A.s_y = p->s_y;
  A.s_out = p->s_out;
  A.err = c->mlp_err;
  A.wait_limit = c->wait_limit;
  A.test_timeout = c->test_timeout;
  int err = 0;
  rc = SGPU_OK;
  if (cudaMemcpyAsync(dx, x, (size_t)n * MLP_IN * sizeof(float), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    rc = SGPU_E_CUDA;
  if (!rc) {
    const long long tiles = (n + MLP_ROWS - 1) / MLP_ROWS;
    k_sgs_mlp<<<(int)std::min<long long>(tiles, 148 * 4), 128, MLP_SMEM_LAUNCH, c->stream>>>(A);
    c->launches++;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(y, dy, (size_t)n * MLP_OUT * sizeof(float), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaMemcpyAsync(&err, c->mlp_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
      rc = SGPU_E_CUDA;
  }
  cudaFree(dx);
  cudaFree(dy);
  if (!rc && err) {
    fprintf(stderr, "simson_b200: sgpu_sgs_mlp_eval: tensor-core wait timed out\n");
    rc = SGPU_E_TIMEOUT;
  }
  return rc;
}
