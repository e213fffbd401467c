// Host build of the pencil algebra of step 3 (the same source the kernels
// run), exported for the CPU unit tests that compare it with the
// reference's setmacrhs/trid/dcheb.  Not part of the device library.
#include <cstring>
#include <vector>

#include "fft.cuh"
#include "cheb_tc.cuh"
#include "les.cuh"
#include "les_filter.h"
#include "step3.cuh"

using namespace sb;

extern "C" void sbh_tau_solve(double lam, int n, int m, const double* f, double* x, const double* bc1,
                              const double* bc2, double* cp, double* wt) {
  // columns are contiguous vectors of n doubles; m <= 5
  Col F[5], X[5];
  for (int q = 0; q < m; ++q) {
    F[q] = Col{const_cast<double*>(f) + (size_t)q * n, 1};
    X[q] = Col{x + (size_t)q * n, 1};
  }
  Col C{cp, 1}, W{wt, 1};
  switch (m) {
    case 1: tau_solve<1>(lam, n, F, X, bc1, bc2, C, W); break;
    case 2: tau_solve<2>(lam, n, F, X, bc1, bc2, C, W); break;
    case 3: tau_solve<3>(lam, n, F, X, bc1, bc2, C, W); break;
    case 4: tau_solve<4>(lam, n, F, X, bc1, bc2, C, W); break;
    default: tau_solve<5>(lam, n, F, X, bc1, bc2, C, W); break;
  }
}

extern "C" void sbh_cheb_deriv(const double* a, double* b, int n) {
  cheb_deriv(Col{b, 1}, Col{const_cast<double*>(a), 1}, n);
}

// Host run of the shared-memory FFT passes on B interleaved columns
// (element i of column b at [i*B + b]); in/out complex interleaved.
extern "C" int sbh_fft(int n, const double* in, double* out, int sign) {
  const FFTPlan plan = fft_make_plan(n);
  if (plan.npass < 0) return -1;
  double2* tw = new double2[n];
  for (int m = 0; m < n; ++m) {
    long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
    tw[m] = double2{(double)cosl(ang), (double)sinl(ang)};
  }
  double2* a = new double2[n];
  double2* b = new double2[n];
  for (int i = 0; i < n; ++i) a[i] = double2{in[2 * i], in[2 * i + 1]};
  double2* src = a;
  double2* dst = b;
  for (int p = 0; p < plan.npass; ++p) {
    fft_pass<double, 1>(src, dst, plan, p, tw, sign, 0, 1);
    double2* t = src;
    src = dst;
    dst = t;
  }
  for (int i = 0; i < n; ++i) {
    out[2 * i] = src[i].x;
    out[2 * i + 1] = src[i].y;
  }
  delete[] a;
  delete[] b;
  delete[] tw;
  return plan.npass;
}

// ADM-RT filter tables (les_filter.h) for the CPU comparison with the
// reference's init_filter: g1, g2 [nyp][5], specx [nx/2+1], specz [nz/2+1],
// lpfxz [nz][nx/2].  Returns 0, or -1 if the tables cannot be built.
extern "C" int sbh_les_filter(int nyp, int nx, int nz, double cutoff, int iord, double* g1, double* g2, double* specx,
                              double* specz, double* lpfxz) {
  LesFilter F;
  if (!les_filter_build(nyp, nx, nz, cutoff, iord, F)) return -1;
  memcpy(g1, F.g1.data(), F.g1.size() * sizeof(double));
  memcpy(g2, F.g2.data(), F.g2.size() * sizeof(double));
  memcpy(specx, F.specx.data(), F.specx.size() * sizeof(double));
  memcpy(specz, F.specz.data(), F.specz.size() * sizeof(double));
  memcpy(lpfxz, F.lpfxz.data(), F.lpfxz.size() * sizeof(double));
  return 0;
}

// The secondary filter of the dynamic HPF model (les_filter_build with
// secondary = true): g1, g2 [nyp][5], lpfxz, filtxz [nz][nx/2].
extern "C" int sbh_les_filter2(int nyp, int nx, int nz, double cutoff, int iord, double* g1, double* g2,
                               double* lpfxz, double* filtxz) {
  LesFilter F;
  if (!les_filter_build(nyp, nx, nz, cutoff, iord, F, true)) return -1;
  memcpy(g1, F.g1.data(), F.g1.size() * sizeof(double));
  memcpy(g2, F.g2.data(), F.g2.size() * sizeof(double));
  memcpy(lpfxz, F.lpfxz.data(), F.lpfxz.size() * sizeof(double));
  memcpy(filtxz, F.filtxz.data(), F.filtxz.size() * sizeof(double));
  return 0;
}

// One high-pass filtered column (the device routine run on the host):
// in/out complex interleaved, nyp values; mode = ihighorder.
extern "C" int sbh_les_hpf_column(int nyp, int nx, int nz, double cutoff, int iord, int mode, int kx, int iz,
                                  const double* in, double* out) {
  LesFilter F;
  if (!les_filter_build(nyp, nx, nz, cutoff, iord, F)) return -1;
  std::vector<double> coef;
  les_filter_rows(F, coef);
  YFilter Y{coef.data(), F.fact2, F.factm2, nyp};
  std::vector<double2> src(nyp), gu(nyp), Z(nyp);
  for (int j = 0; j < nyp; ++j) src[j] = double2{in[2 * j], in[2 * j + 1]};
  const size_t t = (size_t)iz * F.nx2 + kx;
  les_hpf_column(Y, mode, iord, F.lpfxz[t], F.filtxz[t], src.data(), gu.data(), Z.data(), 1);
  for (int j = 0; j < nyp; ++j) {
    out[2 * j] = gu[j].x;
    out[2 * j + 1] = gu[j].y;
  }
  return 0;
}

// One application of the wall-normal filter (hpf = 1 high pass, 0 low pass)
// to a real column, as the reference's hpf_y / lpf_y on one row.
extern "C" int sbh_les_yfilter(int nyp, double cutoff, int hpf, const double* in, double* out) {
  LesFilter F;
  if (!les_filter_build(nyp, 8, 8, cutoff, 0, F)) return -1;
  std::vector<double> coef;
  les_filter_rows(F, coef);
  YFilter Y{coef.data(), F.fact2, F.factm2, nyp};
  std::vector<double2> Z(nyp);
  yfilter_column(
      Y, hpf != 0, [&](int j) { return double2{in[j], 0.0}; }, Z.data(), 1, [&](int j, double2 x) { out[j] = x.x; });
  return 0;
}

// The reordered-sum variant of the tau solve used by the mixed path, with the
// derivative parity sums; dsum[2*q + 0/1] = sum over even / odd j of (D x_q)_j.
extern "C" void sbh_tau_solve_fast(double lam, int n, int m, const double* f, double* x, const double* bc1,
                                   const double* bc2, double* cp, double* dsum) {
  Col F[5], X[5];
  for (int q = 0; q < m; ++q) {
    F[q] = Col{const_cast<double*>(f) + (size_t)q * n, 1};
    X[q] = Col{x + (size_t)q * n, 1};
  }
  Col C{cp, 1}, W{nullptr, 1};
  double ds[5][2] = {};
  switch (m) {
    case 1: tau_solve<1, double, double, true>(lam, n, F, X, bc1, bc2, C, W, ds); break;
    case 2: tau_solve<2, double, double, true>(lam, n, F, X, bc1, bc2, C, W, ds); break;
    case 3: tau_solve<3, double, double, true>(lam, n, F, X, bc1, bc2, C, W, ds); break;
    case 4: tau_solve<4, double, double, true>(lam, n, F, X, bc1, bc2, C, W, ds); break;
    default: tau_solve<5, double, double, true>(lam, n, F, X, bc1, bc2, C, W, ds); break;
  }
  for (int q = 0; q < m; ++q) {
    dsum[2 * q] = ds[q][0];
    dsum[2 * q + 1] = ds[q][1];
  }
}

// Four interleaved columns (the paired-column passes), FP64 or FP32 (prec 1):
// in/out complex interleaved, element i of column b at [(i*4 + b)].
template <class T>
static int host_fft4(int n, const double* in, double* out, int sign) {
  typedef typename C2<T>::type V;
  const FFTPlan plan = fft_make_plan(n);
  if (plan.npass < 0) return -1;
  std::vector<V> tw(n), a(4 * (size_t)n), b(4 * (size_t)n);
  for (int m = 0; m < n; ++m) {
    long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
    tw[m] = V{(T)cosl(ang), (T)sinl(ang)};
  }
  for (size_t i = 0; i < 4 * (size_t)n; ++i) a[i] = V{(T)in[2 * i], (T)in[2 * i + 1]};
  V* src = a.data();
  V* dst = b.data();
  for (int p = 0; p < plan.npass; ++p) {
    fft_pass<T, 4>(src, dst, plan, p, tw.data(), sign, 0, 1);
    V* t = src;
    src = dst;
    dst = t;
  }
  for (size_t i = 0; i < 4 * (size_t)n; ++i) {
    out[2 * i] = (double)src[i].x;
    out[2 * i + 1] = (double)src[i].y;
  }
  return plan.npass;
}

extern "C" int sbh_fft4(int n, const double* in, double* out, int sign, int prec) {
  return prec ? host_fft4<float>(n, in, out, sign) : host_fft4<double>(n, in, out, sign);
}

// The compile-time plan (cfft) of the fixed transform lengths over B = 3, 4
// or 6 interleaved columns, sequentially on the host; in/out as sbh_fft4.
template <class T, int B, int N>
static int host_cfft(const double* in, double* out, int sign) {
  typedef typename C2<T>::type V;
  std::vector<V> tw(N), a(B * (size_t)N), b(B * (size_t)N);
  for (int m = 0; m < N; ++m) {
    long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)N;
    tw[m] = V{(T)cosl(ang), (T)sinl(ang)};
  }
  for (size_t i = 0; i < B * (size_t)N; ++i) a[i] = V{(T)in[2 * i], (T)in[2 * i + 1]};
  std::vector<V> in2(a), out2(B * (size_t)N), c0(B * (size_t)N), c1(B * (size_t)N);
  V* res = sign > 0 ? cfft<T, B, N, 1, 1>(a.data(), b.data(), tw.data(), 0)
                    : cfft<T, B, N, -1, 1>(a.data(), b.data(), tw.data(), 0);
  // the accessor form (first pass reads the input array, last pass writes the
  // output array) must give the same bits
  SmemLd<T, B> ld{in2.data()};
  SmemSt<T, B> st{out2.data()};
  if (sign > 0)
    cfft_io<T, B, N, 1, 1>(ld, st, c0.data(), c1.data(), tw.data(), 0);
  else
    cfft_io<T, B, N, -1, 1>(ld, st, c0.data(), c1.data(), tw.data(), 0);
  for (size_t i = 0; i < B * (size_t)N; ++i) {
    if (memcmp(&out2[i], &res[i], sizeof(V)) != 0) return -2;
    out[2 * i] = (double)res[i].x;
    out[2 * i + 1] = (double)res[i].y;
  }
  return cplan_make(N).npass;
}

template <class T, int N>
static int host_cfft_b(int cols, const double* in, double* out, int sign) {
  switch (cols) {
    case 3: return host_cfft<T, 3, N>(in, out, sign);
    case 4: return host_cfft<T, 4, N>(in, out, sign);
    case 6: return host_cfft<T, 6, N>(in, out, sign);
    default: return -1;
  }
}

extern "C" int sbh_cfft(int n, int cols, const double* in, double* out, int sign, int prec) {
  switch (n) {
#define SB_CASE(N) \
  case N: return prec ? host_cfft_b<float, N>(cols, in, out, sign) : host_cfft_b<double, N>(cols, in, out, sign);
    SB_CASE(72) SB_CASE(96) SB_CASE(240) SB_CASE(288) SB_CASE(576)
#undef SB_CASE
    default: return -1;
  }
}

// The tensor-core Chebyshev transform emulated on the host in FP64 from its
// matrix image: the even/odd folding of the input, the two half-matrix
// products with hi + lo decoded from the tile layout, and the unfolding --
// the kernel's arithmetic without the TF32 split of the data.  in/out: n rows
// of ncol values.  Returns the chunk count, or -1 if an image entry is not a
// TF32 value.
extern "C" int sbh_chb_apply(int n, int inverse, double scale, int ncol, const double* in, double* out) {
  std::vector<unsigned char> img;
  chb_build_matrix(n, inverse, scale, img);
  const int N = n - 1, H = N / 2, ne = chb_even_chunks(n), no = chb_odd_chunks(n);
  const int KE = ne * CHB_KC, KO = no * CHB_KC;
  std::vector<double> Me((size_t)CHB_NMAX * KE, 0.0), Mo((size_t)CHB_NMAX * (KO > 0 ? KO : 1), 0.0);
  for (int q = 0; q < ne + no; ++q) {
    const bool odd = chb_is_odd(q, no);
    const int pi = chb_part_index(q);
    const unsigned char* base = img.data() + (size_t)q * CHB_CHUNK_BYTES;
    for (int r = 0; r < CHB_NMAX; ++r)
      for (int kk = 0; kk < CHB_KC; ++kk) {
        float hi, lo;
        memcpy(&hi, base + chb_canon(r, kk), 4);
        memcpy(&lo, base + CHB_A_BYTES + chb_canon(r, kk), 4);
        unsigned uh, ul;
        memcpy(&uh, &hi, 4);
        memcpy(&ul, &lo, 4);
        if ((uh & 0x1FFFu) || (ul & 0x1FFFu)) return -1;
        const int c = pi * CHB_KC + kk;
        (odd ? Mo[(size_t)r * KO + c] : Me[(size_t)r * KE + c]) = (double)hi + (double)lo;
      }
  }
  std::vector<double> ev(KE), od(KO > 0 ? KO : 1), E(CHB_NMAX), O(CHB_NMAX);
  for (int col = 0; col < ncol; ++col) {
    auto x = [&](int row) { return in[(size_t)row * ncol + col]; };
    for (int m = 0; m < KE; ++m)
      ev[m] = inverse ? (m <= H ? x(2 * m) : 0.0) : (m < H ? x(m) + x(N - m) : (m == H ? x(H) : 0.0));
    for (int m = 0; m < KO; ++m) od[m] = m < H ? (inverse ? x(2 * m + 1) : x(m) - x(N - m)) : 0.0;
    for (int r = 0; r < CHB_NMAX; ++r) {
      double se = 0.0, so = 0.0;
      for (int c = 0; c < KE; ++c) se += Me[(size_t)r * KE + c] * ev[c];
      for (int c = 0; c < KO; ++c) so += Mo[(size_t)r * KO + c] * od[c];
      E[r] = se;
      O[r] = so;
    }
    auto y = [&](int row) -> double& { return out[(size_t)row * ncol + col]; };
    if (!inverse) {
      for (int m = 0; m <= H; ++m) y(2 * m) = E[m];
      for (int m = 0; m < H; ++m) y(2 * m + 1) = O[m];
    } else {
      for (int j = 0; j < H; ++j) {
        y(j) = E[j] + O[j];
        y(N - j) = E[j] - O[j];
      }
      y(H) = E[H];
    }
  }
  return ne + no;
}
