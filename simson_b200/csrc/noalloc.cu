// sgpu_nonlin_noalloc: the nonlinear step (step 2, H = u x omega and the CFL
// partial maximum) for callers that must not allocate device memory.
//
// Who needs it: hosts that own every device buffer themselves and forbid the
// solver library from calling cudaMalloc -- e.g. a Fortran/OpenACC code whose
// device memory is managed by its own pool, or a host that has already
// reserved (nearly) all of the GPU's memory for its fields.  Such a caller
// passes its own device input and output arrays and gets the same kernels as
// sgpu_nonlin, with the two intermediate buffers of the step (the z-transformed
// fields and the x-transformed products) and the small tables (twiddles,
// wavenumbers, CFL grid spacing) placed in one file-scope static device array.
//
// Limits and sharing rules:
//   * the array is SGPU_NOALLOC_SCRATCH_BYTES (64 MiB) of intermediates plus
//     SGPU_NOALLOC_TABLE_BYTES of tables; every GPU that loads the library
//     holds it until the process exits;
//   * grids whose intermediates need more (9*ny*(3nz/2)*(nx/2) complex doubles)
//     are rejected with SGPU_E_PARAM and a message on stderr; so are
//     precision != SGPU_FP64 (the arrays are complex doubles) and the LES
//     models (this entry point forms H = u x omega only);
//   * every call uses the same array and leaves its contents behind; calls that
//     overlap on the GPU (different streams, or different host threads on the
//     same device) race on it and must be serialised by the caller;
//   * every call looks up the array's device address (cudaGetSymbolAddress)
//     with the caller's device current, so a device reset or another context
//     on the same device never sees a stale address; the first lookup on a
//     device may load the library's device code, so make the first call on a
//     device before any stream capture;
//   * every call copies its small tables (twiddles, wavenumbers, CFL spacing)
//     from host memory into the array and, when cflp_max is given, waits for
//     the stream to read the CFL maximum back.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/simson_b200.h"
#include "fft.cuh"
#include "layout.cuh"
#include "step2.cuh"

using namespace sb;

#define SGPU_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define SGPU_NOALLOC_TABLE_BYTES (512ull << 10)
#define SGPU_NOALLOC_MAX_FFT 8192
#define SGPU_NOALLOC_MAX_MODES 4096

static __device__ __align__(256) unsigned char g_noalloc_area[SGPU_NOALLOC_SCRATCH_BYTES + SGPU_NOALLOC_TABLE_BYTES];

namespace {

// The host-side name of the static array is a stand-in, not a device
// address: the device address is looked up on every call, with the caller's
// device current (cheap, and it allocates nothing).
int area_for_current_device(unsigned char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_area);
  if (e != cudaSuccess || p == nullptr) {
    fprintf(stderr, "simson_b200: sgpu_nonlin_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
    return SGPU_E_CUDA;
  }
  *out = static_cast<unsigned char*>(p);
  return SGPU_OK;
}

}  // namespace

extern "C" int sgpu_nonlin_noalloc(const sgpu_params* prm, const void* fields_in, void* h_out, double* cflp_max,
                                   void* stream) {
  if (!prm || !fields_in || !h_out) return SGPU_E_PARAM;
  const sgpu_params& P = *prm;
  if (P.nx < 4 || P.nz < 4 || P.nx % 4 || P.nz % 2 || P.ny < 9 || (P.ny % 2) == 0 || !(P.xl > 0) || !(P.zl > 0))
    return SGPU_E_PARAM;
  if (P.precision != SGPU_FP64) {
    fprintf(stderr, "simson_b200: sgpu_nonlin_noalloc: only precision SGPU_FP64 (complex double arrays)\n");
    return SGPU_E_PARAM;
  }
  Dims g{};
  g.nx = P.nx; g.ny = P.ny; g.nz = P.nz;
  g.nx2 = P.nx / 2; g.nyp = P.ny;
  g.nxp = P.nx + P.nx / 2; g.nzp = P.nz + P.nz / 2;
  g.NP = P.nz * g.nx2; g.zodd = P.nz / 2;
  g.y0 = 0; g.y1 = g.nyp; g.p0 = 0; g.p1 = g.NP;  // the whole domain
  const size_t fine = (size_t)g.nyp * g.nzp * g.nx2 * sizeof(double2);
  const size_t need = 9 * fine;
  if (need > SGPU_NOALLOC_SCRATCH_BYTES || g.nzp > SGPU_NOALLOC_MAX_FFT || g.nxp > SGPU_NOALLOC_MAX_FFT ||
      g.nx2 > SGPU_NOALLOC_MAX_MODES || g.nz > SGPU_NOALLOC_MAX_MODES || g.nyp > SGPU_NOALLOC_MAX_MODES) {
    fprintf(stderr,
            "simson_b200: sgpu_nonlin_noalloc: grid %dx%dx%d needs %zu bytes of intermediates; the static area "
            "holds %llu (use sgpu_nonlin)\n",
            P.nx, P.ny, P.nz, need, (unsigned long long)SGPU_NOALLOC_SCRATCH_BYTES);
    return SGPU_E_PARAM;
  }
  const FFTPlan pz = fft_make_plan(g.nzp), px = fft_make_plan(g.nxp);
  if (pz.npass < 0 || px.npass < 0) return SGPU_E_PARAM;
  unsigned char* area = nullptr;
  int rc = area_for_current_device(&area);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  // carve the area: intermediates, then tables (each 256-byte aligned)
  double2* zb = reinterpret_cast<double2*>(area);
  double2* xb = zb + 6 * (size_t)g.nyp * g.nzp * g.nx2;
  unsigned char* tab = area + SGPU_NOALLOC_SCRATCH_BYTES;
  double2* twz = reinterpret_cast<double2*>(tab);
  double2* twx = twz + SGPU_NOALLOC_MAX_FFT;
  double* alfa = reinterpret_cast<double*>(twx + SGPU_NOALLOC_MAX_FFT);
  double* beta = alfa + SGPU_NOALLOC_MAX_MODES;
  double* dyi = beta + SGPU_NOALLOC_MAX_MODES;
  unsigned long long* cfl_bits = reinterpret_cast<unsigned long long*>(dyi + SGPU_NOALLOC_MAX_MODES);

  // tables on the host stack (no allocation), packed as they sit in the area
  // and copied with one call; the same formulas as sgpu_init so the results
  // match sgpu_nonlin bit for bit
  {
    static_assert(sizeof(double2) * 2 * SGPU_NOALLOC_MAX_FFT + sizeof(double) * 3 * SGPU_NOALLOC_MAX_MODES <=
                      SGPU_NOALLOC_TABLE_BYTES - 256,
                  "tables exceed their part of the area");
    constexpr size_t kTab = sizeof(double2) * 2 * SGPU_NOALLOC_MAX_FFT + sizeof(double) * 3 * SGPU_NOALLOC_MAX_MODES;
    // one static host block for every caller, held under a lock while it is
    // filled and staged by the copy below
    alignas(16) static unsigned char host_tab[kTab];
    static std::mutex host_tab_lock;
    std::lock_guard<std::mutex> lock(host_tab_lock);
    double2* htwz = reinterpret_cast<double2*>(host_tab);
    double2* htwx = htwz + SGPU_NOALLOC_MAX_FFT;
    double* halfa = reinterpret_cast<double*>(htwx + SGPU_NOALLOC_MAX_FFT);
    double* hbeta = halfa + SGPU_NOALLOC_MAX_MODES;
    double* hdyi = hbeta + SGPU_NOALLOC_MAX_MODES;
    for (int pass = 0; pass < 2; ++pass) {
      const int n = pass ? g.nxp : g.nzp;
      double2* tw = pass ? htwx : htwz;
      for (int m = 0; m < n; ++m) {
        long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
        tw[m] = double2{(double)cosl(ang), (double)sinl(ang)};
      }
    }
    const double pi = 3.1415926535897932385;
    for (int x = 0; x < g.nx2; ++x) halfa[x] = 2. * pi / P.xl * (double)x;
    for (int z = 0; z < g.nz; ++z) hbeta[z] = 0.0;
    for (int z = 1; z <= g.nz / 2; ++z) {
      hbeta[z] = 2. * pi / P.zl * (double)z;
      hbeta[g.nz - z] = -2. * pi / P.zl * (double)z;
    }
    double eta[SGPU_NOALLOC_MAX_MODES], deta[SGPU_NOALLOC_MAX_MODES];
    for (int y = 0; y < g.nyp; ++y) eta[y] = cos(pi * (double)y / (double)(g.nyp - 1));
    deta[0] = 1. - eta[1];
    deta[g.nyp - 1] = deta[0];
    for (int y = 1; y < g.nyp - 1; ++y) deta[y] = (eta[y - 1] - eta[y + 1]) * .5;
    for (int y = 0; y < g.nyp; ++y) {
      double d = (double)(g.ny - 1) / (double)(g.nyp - 1) / deta[y];
      if (g.ny >= 17) d = fmin(d, (double)(g.ny - 1) * (double)(g.ny - 1) / 10. / 3.14);
      hdyi[y] = d;
    }
    // a copy from pageable memory: it returns once the block is staged, so the
    // block may be refilled after it
    if (cudaMemcpyAsync(twz, host_tab, kTab, cudaMemcpyHostToDevice, st) != cudaSuccess) return SGPU_E_CUDA;
  }
  // the CFL word starts at zero every call
  if (cudaMemsetAsync(cfl_bits, 0, sizeof(unsigned long long), st) != cudaSuccess) return SGPU_E_CUDA;

  constexpr int KB = 4, RB = 1, TH = 128;
  const size_t s_z = 2 * (size_t)g.nzp * KB * sizeof(double2);
  const size_t s_x = 2 * (size_t)g.nxp * 3 * RB * sizeof(double2);
  if (s_z > 227 * 1024 || s_x > 227 * 1024) return SGPU_E_PARAM;
  if (cudaFuncSetAttribute(k_zinv<double, KB, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s_z) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_zfwd<double, KB, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s_z) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_xpass<double, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s_x) !=
          cudaSuccess) {
    fprintf(stderr, "simson_b200: sgpu_nonlin_noalloc: shared-memory opt-in refused: %s\n",
            cudaGetErrorString(cudaGetLastError()));
    return SGPU_E_CUDA;
  }
  const double2* in = static_cast<const double2*>(fields_in);
  double2* out = static_cast<double2*>(h_out);
  dim3 gz((g.nx2 + KB - 1) / KB, g.nyp);
  k_zinv<double, KB, double><<<gz, TH, s_z, st>>>(in, zb, g, pz, twz, alfa, beta, 0);
  dim3 gx((g.nzp + RB - 1) / RB, g.nyp);
  const double dxi = (double)(g.nx - 2) / P.xl;
  const double dzi = (double)(g.nz - 2) / P.zl;
  k_xpass<double, RB><<<gx, TH, s_x, st>>>(zb, xb, g, px, twx, dyi, dxi, dzi, P.rot, cfl_bits, nullptr,
                                          Fringe{nullptr, nullptr});
  k_zfwd<double, KB, double><<<gz, TH, s_z, st>>>(xb, out, g, pz, twz, nullptr, 0.0);
  if (cudaGetLastError() != cudaSuccess) return SGPU_E_CUDA;
  if (cflp_max) {
    unsigned long long bits = 0;
    if (cudaMemcpyAsync(&bits, cfl_bits, sizeof(bits), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return SGPU_E_CUDA;
    memcpy(cflp_max, &bits, sizeof(double));
  }
  return SGPU_OK;
}
