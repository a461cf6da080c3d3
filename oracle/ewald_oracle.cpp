// ewald_oracle.cpp -- TEST INFRASTRUCTURE, NOT THE PRODUCT.
//
// CPU restatement of the reference's fast 3D Ewald library and of DFTB+'s
// stock Ewald stress.  Loop order, OpenMP partitioning and the parameter chain
// follow the Fortran sources cited beside each function (paths relative to the
// reference project).  The only deliberate difference: FFTW3, which is not in
// this image, is replaced by a plain recursive mixed-radix DFT with the same
// sign convention and no normalisation (nfft/fft_backend.f90:43-58).
//
// parity unpinned: the reference has no tests or golden vectors for this path
// and cannot be built here (see ewald_oracle.h).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg load
// this library; the CUDA product never links or calls it.

#include "ewald_oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cplx = std::complex<double>;

// common/ewald_constants.f90:10-15
const double kPi = std::acos(-1.0);
const double kSqrtPi = std::sqrt(kPi);

// common/ewald_validation.f90:13-20
constexpr double kMinSeparationSquared = 1.0e-24;
constexpr double kMinWavenumberSquared = 1.0e-24;
constexpr double kNeutralityTolerance = 1.0e-8;
// common/ewald_geometry.f90:20
constexpr double kMinVolume = 1.0e-18;
// nfft/nfft.f90:43 and :49
constexpr int kOversampling = 2;
const double kWindowErrorRate = 2.0 * kPi / 3.0;
// nfft/fft_backend.f90:29
constexpr int kMinTransformLength = 4;
// fft/ewald_fft_3d_parameters.f90:16-21
constexpr double kRealCutoffPrefactor = 3.0;
constexpr double kRealCutoffBudgetFraction = 0.2;
// common/ewald_cell_list.f90:27
constexpr int kMinBoxesPerAxis = 3;
// common/accuracy.F90:114 (stock DFTB+ searches)
constexpr int kNSearchIter = 30;

inline int fmodulo(int a, int n) {  // Fortran modulo(a, n) for n > 0
  int r = a % n;
  return r < 0 ? r + n : r;
}
inline int ffloor(double x) { return static_cast<int>(std::floor(x)); }
inline int fceiling(double x) { return static_cast<int>(std::ceil(x)); }

// ----------------------------------------------------------------------------
// Geometry: common/ewald_geometry.f90:22-93
// ----------------------------------------------------------------------------
struct Cell {
  double lat[3][3];  // lat[i][d]: lattice vector a_i, component d
  double rec[3][3];  // rec[i][d]: dual vector b_i (no 2 pi)
  double volume;
  double latLen[3], recLen[3];
};

void cross(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// cell_metrics_3d, common/ewald_geometry.f90:65-93.  `lat` is Fortran
// latVecs(3,3) with rows = vectors, column-major storage.
int cell_metrics(const double* latFortran, Cell& cell) {
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) cell.lat[i][d] = latFortran[i + 3 * d];
  double c23[3];
  cross(cell.lat[1], cell.lat[2], c23);
  cell.volume = std::fabs(cell.lat[0][0] * c23[0] + cell.lat[0][1] * c23[1] + cell.lat[0][2] * c23[2]);
  if (cell.volume <= kMinVolume) return EWO_ERR_VOLUME;
  double c31[3], c12[3];
  cross(cell.lat[2], cell.lat[0], c31);
  cross(cell.lat[0], cell.lat[1], c12);
  for (int d = 0; d < 3; ++d) {
    cell.rec[0][d] = c23[d] / cell.volume;
    cell.rec[1][d] = c31[d] / cell.volume;
    cell.rec[2][d] = c12[d] / cell.volume;
  }
  for (int i = 0; i < 3; ++i) {
    cell.latLen[i] = std::sqrt(cell.lat[i][0] * cell.lat[i][0] + cell.lat[i][1] * cell.lat[i][1] +
                               cell.lat[i][2] * cell.lat[i][2]);
    cell.recLen[i] = std::sqrt(cell.rec[i][0] * cell.rec[i][0] + cell.rec[i][1] * cell.rec[i][1] +
                               cell.rec[i][2] * cell.rec[i][2]);
  }
  return EWO_OK;
}

// check_configuration, common/ewald_validation.f90:26-48
int check_configuration(int n, const double* positions, const double* charges) {
  if (n <= 0) return EWO_ERR_NPARTICLE;
  if (!positions || !charges) return EWO_ERR_ARG;
  double net = 0.0, absolute = 0.0;
  for (int i = 0; i < n; ++i) net += charges[i];
  for (int i = 0; i < n; ++i) absolute += std::fabs(charges[i]);
  if (std::fabs(net) > kNeutralityTolerance * absolute) return EWO_ERR_NOT_NEUTRAL;
  return EWO_OK;
}

// lambert_w0, common/ewald_lambert_w.f90:27-56 (Halley iteration)
double lambert_w0(double x) {
  if (x <= 0.0) return 0.0;
  double w = std::log(1.0 + x);
  for (int it = 1; it <= 60; ++it) {
    double ew = std::exp(w);
    double residual = w * ew - x;
    double wp1 = w + 1.0;
    double corr = residual / (ew * wp1 - 0.5 * (w + 2.0) * residual / wp1);
    w = w - corr;
    if (std::fabs(corr) <= 1.0e-15 * (1.0 + std::fabs(w))) break;
  }
  return w;
}

// splitting_from_real_budget, common/ewald_truncation.f90:53-78
double splitting_from_real_budget(double r_cut, double q2sum, int n, double volume, double budget) {
  double argument = (2.0 / budget) * q2sum * std::sqrt(r_cut / (static_cast<double>(n) * volume));
  double w;
  if (argument > 0.0)
    w = lambert_w0(argument);
  else
    w = -std::log(budget);
  if (w <= 0.0) w = -std::log(budget);
  return std::sqrt(w) / r_cut;
}

// cutoff_from_fourier_budget, common/ewald_truncation.f90:84-104
double cutoff_from_fourier_budget(double q2sum, int n, double edge, double alpha, double budget) {
  double argument = (4.0 / (3.0 * edge * edge)) *
                    std::pow(2.0 / (static_cast<double>(n) * alpha * kPi), 2.0 / 3.0) *
                    std::pow(2.0 * q2sum / budget, 4.0 / 3.0);
  double w = lambert_w0(argument);
  if (w <= 0.0) w = -std::log(budget);
  return std::sqrt(3.0) * alpha * std::sqrt(w);
}

// next_fast_length, nfft/fft_backend.f90:73-91
int next_fast_length(int n) {
  int m = std::max(n, 2);
  if (m % 2 != 0) m += 1;
  for (;;) {
    int r = m;
    while (r % 2 == 0) r /= 2;
    while (r % 3 == 0) r /= 3;
    while (r % 5 == 0) r /= 5;
    while (r % 7 == 0) r /= 7;
    if (r == 1) break;
    m += 2;
  }
  return m;
}

// window_shape, nfft/nfft.f90:82-92
double window_shape(int m) {
  return (2.0 * kOversampling / (2.0 * kOversampling - 1.0)) * (static_cast<double>(m) / kPi);
}

// window_cutoff_from_budget, nfft/nfft.f90:99-109
int window_cutoff_from_budget(double budget) {
  return std::max(2, fceiling(std::log(4.0 / budget) / kWindowErrorRate));
}

// modes_along_axis, fft/ewald_fft_3d_parameters.f90:152-168
int modes_along_axis(double k_cut, double len) {
  int highest = fceiling(k_cut * len / (2.0 * kPi)) + 1;
  return std::max(next_fast_length(2 * highest), kMinTransformLength);
}

// choose_parameters, fft/ewald_fft_3d_parameters.f90:52-142
int choose_parameters(const Cell& cell, double q2sum, int n, double tol, const ewo_overrides* ov,
                      ewo_params& p) {
  ewo_overrides none{};
  if (!ov) ov = &none;
  double meanSpacing = std::pow(cell.volume / static_cast<double>(n), 1.0 / 3.0);
  if (ov->has_r_cut) {
    p.r_cut = ov->r_cut;
  } else if (ov->has_alpha) {
    p.r_cut = std::sqrt(-std::log(tol)) / ov->alpha;
  } else {
    p.r_cut = kRealCutoffPrefactor * meanSpacing;
    double maxRec = std::max(cell.recLen[0], std::max(cell.recLen[1], cell.recLen[2]));
    double cellListLimit = 0.999 / (3.0 * maxRec);
    if (cellListLimit >= 1.5 * meanSpacing) p.r_cut = std::min(p.r_cut, cellListLimit);
  }
  if (ov->has_alpha)
    p.alpha = ov->alpha;
  else
    p.alpha = splitting_from_real_budget(p.r_cut, q2sum, n, cell.volume,
                                         kRealCutoffBudgetFraction * tol);
  if (p.alpha <= 0.0) return EWO_ERR_ALPHA;
  p.k_cut = cutoff_from_fourier_budget(q2sum, n, std::pow(cell.volume, 1.0 / 3.0), p.alpha, tol);
  if (ov->has_k_cut) p.k_cut = ov->k_cut;
  p.window_cutoff = window_cutoff_from_budget(tol);
  if (ov->has_window_cutoff) p.window_cutoff = ov->window_cutoff;
  for (int a = 0; a < 3; ++a) p.n_modes[a] = modes_along_axis(p.k_cut, cell.latLen[a]);
  if (ov->has_n_modes)
    for (int a = 0; a < 3; ++a) p.n_modes[a] = ov->n_modes;
  return EWO_OK;
}

// ----------------------------------------------------------------------------
// FFT replacement for FFTW (nfft/fft_backend.f90:43-58): unnormalised complex
// DFT, isign >= 0 means exp(+2 pi i jk/n) (FFTW_BACKWARD), isign < 0 means
// exp(-2 pi i jk/n) (FFTW_FORWARD).  Recursive decimation in time over the
// prime factors of n.
// ----------------------------------------------------------------------------
struct Plan1 {
  int n = 0;
  std::vector<int> factors;  // radix, remaining length pairs
  std::vector<cplx> tw;      // tw[k] = exp(sign * 2 pi i k / n)
};

Plan1 make_plan(int n, int isign) {
  Plan1 p;
  p.n = n;
  int rem = n;
  while (rem > 1) {
    int r;
    if (rem % 4 == 0)
      r = 4;
    else if (rem % 2 == 0)
      r = 2;
    else if (rem % 3 == 0)
      r = 3;
    else if (rem % 5 == 0)
      r = 5;
    else if (rem % 7 == 0)
      r = 7;
    else {
      r = 11;
      while (rem % r != 0) r += 2;
    }
    rem /= r;
    p.factors.push_back(r);
    p.factors.push_back(rem);
  }
  p.tw.resize(n);
  double s = isign >= 0 ? 1.0 : -1.0;
  for (int k = 0; k < n; ++k) {
    double ang = 2.0 * kPi * static_cast<double>(k) / static_cast<double>(n);
    p.tw[k] = cplx(std::cos(ang), s * std::sin(ang));
  }
  return p;
}

void fft_rec(cplx* out, const cplx* in, int fstride, int istride, const int* factors, const Plan1& p) {
  const int radix = factors[0];
  const int m = factors[1];
  if (m == 1) {
    for (int k = 0; k < radix; ++k) out[k] = in[static_cast<long>(k) * fstride * istride];
  } else {
    for (int k = 0; k < radix; ++k)
      fft_rec(out + k * m, in + static_cast<long>(k) * fstride * istride, fstride * radix, istride,
              factors + 2, p);
  }
  // Combine: X[u + s m] = sum_q W_n^{q u} W_radix^{q s} Y_q[u]
  cplx scratch[64];
  std::vector<cplx> big;
  cplx* sc = scratch;
  if (radix > 64) {
    big.resize(radix);
    sc = big.data();
  }
  const int n = p.n;
  for (int u = 0; u < m; ++u) {
    for (int q = 0; q < radix; ++q) {
      long e = (static_cast<long>(q) * u * fstride) % n;
      sc[q] = out[q * m + u] * p.tw[e];
    }
    for (int s = 0; s < radix; ++s) {
      cplx acc = sc[0];
      for (int q = 1; q < radix; ++q) {
        long e = (static_cast<long>(q) * s * m * fstride) % n;
        acc += sc[q] * p.tw[e];
      }
      out[s * m + u] = acc;
    }
  }
}

void fft_line(const Plan1& p, const cplx* in, long stride, cplx* out) {
  if (p.n == 1) {
    out[0] = in[0];
    return;
  }
  fft_rec(out, in, 1, static_cast<int>(stride), p.factors.data(), p);
}

// fft_3d_inplace, nfft/fft_backend.f90:43-58: Fortran order, i1 fastest.
void fft3d(cplx* grid, int n1, int n2, int n3, int isign) {
  const int ns[3] = {n1, n2, n3};
  const long strides[3] = {1, static_cast<long>(n1), static_cast<long>(n1) * n2};
  for (int axis = 0; axis < 3; ++axis) {
    const int n = ns[axis];
    if (n == 1) continue;
    Plan1 plan = make_plan(n, isign);
    const int oa = (axis + 1) % 3, ob = (axis + 2) % 3;
    const long nlines = static_cast<long>(ns[oa]) * ns[ob];
#pragma omp parallel
    {
      std::vector<cplx> line(n), res(n);
#pragma omp for schedule(static)
      for (long l = 0; l < nlines; ++l) {
        int ia = static_cast<int>(l % ns[oa]);
        int ib = static_cast<int>(l / ns[oa]);
        cplx* base = grid + ia * strides[oa] + ib * strides[ob];
        for (int k = 0; k < n; ++k) line[k] = base[k * strides[axis]];
        fft_line(plan, line.data(), 1, res.data());
        for (int k = 0; k < n; ++k) base[k * strides[axis]] = res[k];
      }
    }
  }
}

// ----------------------------------------------------------------------------
// NFFT with a Gaussian window: nfft/nfft.f90
// ----------------------------------------------------------------------------
inline int mode_of_bin(int a, int M) { return a >= M / 2 ? a - M : a; }  // :61-75

// stencil_weights, nfft/nfft.f90:122-159
inline void stencil_weights(double t, int n, int m, double b, int& lowest, double* w /* 2m+1 */) {
  double wrapped = t - std::floor(t);
  double scaled = wrapped * static_cast<double>(n);
  lowest = ffloor(scaled);
  double fraction = scaled - static_cast<double>(lowest);
  if (lowest >= n) lowest -= n;
  double pref = 1.0 / std::sqrt(kPi * b);
  for (int o = -m; o <= m; ++o) {
    double d = fraction - static_cast<double>(o);
    w[o + m] = pref * std::exp(-(d * d) / b);
  }
}

// deconvolution_table, nfft/nfft.f90:163-189
void deconvolution_table(int M, int n, double b, std::vector<int>& idx, std::vector<double>& fac) {
  idx.resize(M);
  fac.resize(M);
  for (int a = 0; a < M; ++a) {
    int k = mode_of_bin(a, M);
    idx[a] = fmodulo(k, n);
    double x = kPi * static_cast<double>(k) / static_cast<double>(n);
    fac[a] = std::exp(b * (x * x));
  }
}

// Wall-clock split of the last ewo_fft_potential_force call (seconds): real
// space, spread, FFTs, gathers, everything else (deconvolution, embedding,
// influence weights).  Reported beside the CPU baseline so that a reader can
// bound how much of the timing depends on the FFT used in place of FFTW.
enum { ST_REAL, ST_SPREAD, ST_FFT, ST_GATHER, ST_OTHER, ST_N };
double g_stage_s[ST_N] = {0, 0, 0, 0, 0};
struct StageTimer {
  int st;
  std::chrono::steady_clock::time_point t0;
  explicit StageTimer(int s) : st(s), t0(std::chrono::steady_clock::now()) {}
  ~StageTimer() {
    g_stage_s[st] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

// adjoint_nfft_3d, nfft/nfft.f90:196-305
void adjoint_nfft(int N, const double* t1, const double* t2, const double* t3, const double* q,
                  int M1, int M2, int M3, int m, cplx* Shat) {
  const int n1 = kOversampling * M1, n2 = kOversampling * M2, n3 = kOversampling * M3;
  const double b = window_shape(m);
  std::vector<cplx> grid(static_cast<size_t>(n1) * n2 * n3, cplx(0.0, 0.0));
  double* g = reinterpret_cast<double*>(grid.data());
  const int W = 2 * m + 1;
  // Step 1: spread, atomic updates on the real part (:256-278).
  StageTimer* spread_timer = new StageTimer(ST_SPREAD);
#pragma omp parallel
  {
    std::vector<double> w1(W), w2(W), w3(W);
#pragma omp for schedule(guided)
    for (int j = 0; j < N; ++j) {
      if (q[j] == 0.0) continue;
      int c1, c2, c3;
      stencil_weights(t1[j], n1, m, b, c1, w1.data());
      stencil_weights(t2[j], n2, m, b, c2, w2.data());
      stencil_weights(t3[j], n3, m, b, c3, w3.data());
      for (int o3 = -m; o3 <= m; ++o3) {
        int i3 = fmodulo(c3 + o3, n3);
        for (int o2 = -m; o2 <= m; ++o2) {
          int i2 = fmodulo(c2 + o2, n2);
          double qw = q[j] * w2[o2 + m] * w3[o3 + m];
          for (int o1 = -m; o1 <= m; ++o1) {
            int i1 = fmodulo(c1 + o1, n1);
            size_t idx = (static_cast<size_t>(i3) * n2 + i2) * n1 + i1;
#pragma omp atomic update
            g[2 * idx] += qw * w1[o1 + m];
          }
        }
      }
    }
  }
  delete spread_timer;
  // Step 2: one transform with sign +1 (:282).
  {
    StageTimer t(ST_FFT);
    fft3d(grid.data(), n1, n2, n3, 1);
  }
  // Step 3: keep the low modes and divide out the window (:286-298).
  StageTimer other(ST_OTHER);
  std::vector<int> i1v, i2v, i3v;
  std::vector<double> f1, f2, f3;
  deconvolution_table(M1, n1, b, i1v, f1);
  deconvolution_table(M2, n2, b, i2v, f2);
  deconvolution_table(M3, n3, b, i3v, f3);
  for (int a3 = 0; a3 < M3; ++a3)
    for (int a2 = 0; a2 < M2; ++a2)
      for (int a1 = 0; a1 < M1; ++a1) {
        size_t src = (static_cast<size_t>(i3v[a3]) * n2 + i2v[a2]) * n1 + i1v[a1];
        Shat[(static_cast<size_t>(a3) * M2 + a2) * M1 + a1] = grid[src] * f1[a1] * f2[a2] * f3[a3];
      }
}

// forward_nfft_3d, nfft/nfft.f90:313-404
void forward_nfft(int N, const double* t1, const double* t2, const double* t3, int M1, int M2, int M3,
                  int m, const cplx* fhat, cplx* f) {
  const int n1 = kOversampling * M1, n2 = kOversampling * M2, n3 = kOversampling * M3;
  const double b = window_shape(m);
  StageTimer* embed_timer = new StageTimer(ST_OTHER);
  std::vector<cplx> grid(static_cast<size_t>(n1) * n2 * n3, cplx(0.0, 0.0));
  std::vector<int> i1v, i2v, i3v;
  std::vector<double> f1, f2, f3;
  deconvolution_table(M1, n1, b, i1v, f1);
  deconvolution_table(M2, n2, b, i2v, f2);
  deconvolution_table(M3, n3, b, i3v, f3);
  for (int a3 = 0; a3 < M3; ++a3)
    for (int a2 = 0; a2 < M2; ++a2)
      for (int a1 = 0; a1 < M1; ++a1) {
        size_t dst = (static_cast<size_t>(i3v[a3]) * n2 + i2v[a2]) * n1 + i1v[a1];
        grid[dst] = fhat[(static_cast<size_t>(a3) * M2 + a2) * M1 + a1] * f1[a1] * f2[a2] * f3[a3];
      }
  delete embed_timer;
  {
    StageTimer t(ST_FFT);
    fft3d(grid.data(), n1, n2, n3, -1);
  }
  const int W = 2 * m + 1;
  StageTimer gather_timer(ST_GATHER);
#pragma omp parallel
  {
    std::vector<double> w1(W), w2(W), w3(W);
#pragma omp for schedule(guided)
    for (int j = 0; j < N; ++j) {
      int c1, c2, c3;
      stencil_weights(t1[j], n1, m, b, c1, w1.data());
      stencil_weights(t2[j], n2, m, b, c2, w2.data());
      stencil_weights(t3[j], n3, m, b, c3, w3.data());
      cplx acc(0.0, 0.0);
      for (int o3 = -m; o3 <= m; ++o3) {
        int i3 = fmodulo(c3 + o3, n3);
        for (int o2 = -m; o2 <= m; ++o2) {
          int i2 = fmodulo(c2 + o2, n2);
          double outer = w2[o2 + m] * w3[o3 + m];
          for (int o1 = -m; o1 <= m; ++o1) {
            int i1 = fmodulo(c1 + o1, n1);
            size_t idx = (static_cast<size_t>(i3) * n2 + i2) * n1 + i1;
            acc += w1[o1 + m] * outer * grid[idx];
          }
        }
      }
      f[j] = acc;
    }
  }
}

// ----------------------------------------------------------------------------
// Real-space branches
// ----------------------------------------------------------------------------

// real_space_potential_force, direct/ewald_direct_3d.f90:192-309 (explicit image sum)
int direct_real_space(int N, const double* pos, const double* q, const Cell& cell, double alpha,
                      double r_cut, double* pot, double* force) {
  const double cut2 = r_cut * r_cut;
  int nImg[3];
  for (int d = 0; d < 3; ++d) nImg[d] = fceiling(r_cut * cell.recLen[d]) + 1;
  std::atomic<int> bad{0};
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < N; ++i) {
    double acc = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
    for (int j = 0; j < N; ++j) {
      for (int nx = -nImg[0]; nx <= nImg[0]; ++nx)
        for (int ny = -nImg[1]; ny <= nImg[1]; ++ny)
          for (int nz = -nImg[2]; nz <= nImg[2]; ++nz) {
            if (i == j && nx == 0 && ny == 0 && nz == 0) continue;
            double dx = pos[i] - pos[j] + nx * cell.lat[0][0] + ny * cell.lat[1][0] + nz * cell.lat[2][0];
            double dy = pos[i + N] - pos[j + N] + nx * cell.lat[0][1] + ny * cell.lat[1][1] +
                        nz * cell.lat[2][1];
            double dz = pos[i + 2 * N] - pos[j + 2 * N] + nx * cell.lat[0][2] + ny * cell.lat[1][2] +
                        nz * cell.lat[2][2];
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < kMinSeparationSquared) {
              bad = 1;
              continue;
            }
            if (r2 > cut2) continue;
            double r = std::sqrt(r2);
            double ec = std::erfc(alpha * r);
            acc += q[j] * ec / r;
            if (force) {
              double ff = q[i] * q[j] * (2.0 * alpha / kSqrtPi * std::exp(-alpha * alpha * r2) + ec / r) / r2;
              fx += ff * dx;
              fy += ff * dy;
              fz += ff * dz;
            }
          }
    }
    pot[i] = acc;
    if (force) {
      force[3 * i] = fx;
      force[3 * i + 1] = fy;
      force[3 * i + 2] = fz;
    }
  }
  return bad ? EWO_ERR_COINCIDENT : EWO_OK;
}

// box_counts_3d / box_index, common/ewald_cell_list.f90:56-91
inline int box_index(double frac, int nb) { return std::min(static_cast<int>(frac * nb), nb - 1); }

// potential_force_cell_list, fft/ewald_fft_3d_real.f90:81-187, with
// build_cell_list_3d, common/ewald_cell_list.f90:96-141
int cell_list_real_space(int N, const double* pos, const double* q, const Cell& cell, double alpha,
                         double r_cut, const int nb[3], double* pot, double* force) {
  std::vector<double> f1(N), f2(N), f3(N);
  std::vector<int> head(static_cast<size_t>(nb[0]) * nb[1] * nb[2], 0), next(N + 1, 0);
  for (int i = 0; i < N; ++i) {
    const double p[3] = {pos[i], pos[i + N], pos[i + 2 * N]};
    f1[i] = cell.rec[0][0] * p[0] + cell.rec[0][1] * p[1] + cell.rec[0][2] * p[2];
    f2[i] = cell.rec[1][0] * p[0] + cell.rec[1][1] * p[1] + cell.rec[1][2] * p[2];
    f3[i] = cell.rec[2][0] * p[0] + cell.rec[2][1] * p[1] + cell.rec[2][2] * p[2];
    f1[i] -= std::floor(f1[i]);
    f2[i] -= std::floor(f2[i]);
    f3[i] -= std::floor(f3[i]);
    int ix = box_index(f1[i], nb[0]), iy = box_index(f2[i], nb[1]), iz = box_index(f3[i], nb[2]);
    size_t h = (static_cast<size_t>(iz) * nb[1] + iy) * nb[0] + ix;
    next[i + 1] = head[h];  // 1-based chains, 0 terminates
    head[h] = i + 1;
  }
  const double cut2 = r_cut * r_cut;
  std::atomic<int> bad{0};
#pragma omp parallel for schedule(guided)
  for (int i = 0; i < N; ++i) {
    int ix = box_index(f1[i], nb[0]), iy = box_index(f2[i], nb[1]), iz = box_index(f3[i], nb[2]);
    double acc = 0.0, fa[3] = {0.0, 0.0, 0.0};
    for (int dz = -1; dz <= 1; ++dz) {
      int jz = fmodulo(iz + dz, nb[2]);
      for (int dy = -1; dy <= 1; ++dy) {
        int jy = fmodulo(iy + dy, nb[1]);
        for (int dx = -1; dx <= 1; ++dx) {
          int jx = fmodulo(ix + dx, nb[0]);
          int j1 = head[(static_cast<size_t>(jz) * nb[1] + jy) * nb[0] + jx];
          while (j1 != 0) {
            int j = j1 - 1;
            if (j != i) {
              double d1 = f1[i] - f1[j];
              d1 -= std::round(d1);
              double d2 = f2[i] - f2[j];
              d2 -= std::round(d2);
              double d3 = f3[i] - f3[j];
              d3 -= std::round(d3);
              double sv[3];
              for (int c = 0; c < 3; ++c) sv[c] = d1 * cell.lat[0][c] + d2 * cell.lat[1][c] + d3 * cell.lat[2][c];
              double r2 = sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2];
              if (r2 < kMinSeparationSquared) bad = 1;
              if (r2 <= cut2) {
                double r = std::sqrt(r2);
                double ec = std::erfc(alpha * r);
                acc += q[j] * ec / r;
                double ff = q[i] * q[j] * (2.0 * alpha / kSqrtPi * std::exp(-alpha * alpha * r2) + ec / r) / r2;
                for (int c = 0; c < 3; ++c) fa[c] += ff * sv[c];
              }
            }
            j1 = next[j1];
          }
        }
      }
    }
    pot[i] = acc;
    for (int c = 0; c < 3; ++c) force[3 * i + c] = fa[c];
  }
  return bad ? EWO_ERR_COINCIDENT : EWO_OK;
}

// short_range_potential_force, fft/ewald_fft_3d_real.f90:32-77
int short_range(int N, const double* pos, const double* q, const Cell& cell, double alpha, double r_cut,
                double* pot, double* force, int* used_cell_list) {
  int nb[3];
  for (int d = 0; d < 3; ++d) nb[d] = ffloor(1.0 / (r_cut * cell.recLen[d]));
  int mn = std::min(nb[0], std::min(nb[1], nb[2]));
  if (used_cell_list) *used_cell_list = mn >= kMinBoxesPerAxis;
  if (mn >= kMinBoxesPerAxis) return cell_list_real_space(N, pos, q, cell, alpha, r_cut, nb, pot, force);
  return direct_real_space(N, pos, q, cell, alpha, r_cut, pot, force);
}

// long_range_potential_force, fft/ewald_fft_3d_fourier.f90:28-153
void long_range(int N, const double* pos, const double* q, const Cell& cell, double alpha,
                const int* M, int m, double* pot, double* force) {
  std::vector<double> t1(N), t2(N), t3(N);
  for (int i = 0; i < N; ++i) {
    const double p[3] = {pos[i], pos[i + N], pos[i + 2 * N]};
    t1[i] = cell.rec[0][0] * p[0] + cell.rec[0][1] * p[1] + cell.rec[0][2] * p[2];
    t2[i] = cell.rec[1][0] * p[0] + cell.rec[1][1] * p[1] + cell.rec[1][2] * p[2];
    t3[i] = cell.rec[2][0] * p[0] + cell.rec[2][1] * p[1] + cell.rec[2][2] * p[2];
  }
  const size_t nm = static_cast<size_t>(M[0]) * M[1] * M[2];
  std::vector<cplx> coef(nm);
  adjoint_nfft(N, t1.data(), t2.data(), t3.data(), q, M[0], M[1], M[2], m, coef.data());
  const double prefactor = 4.0 * kPi / cell.volume;
  const double inv4a2 = 1.0 / (4.0 * (alpha * alpha));
  const double twoPi = 2.0 * kPi;
  for (int a3 = 0; a3 < M[2]; ++a3) {
    int k3 = mode_of_bin(a3, M[2]);
    for (int a2 = 0; a2 < M[1]; ++a2) {
      int k2 = mode_of_bin(a2, M[1]);
      for (int a1 = 0; a1 < M[0]; ++a1) {
        int k1 = mode_of_bin(a1, M[0]);
        size_t idx = (static_cast<size_t>(a3) * M[1] + a2) * M[0] + a1;
        if (k1 == 0 && k2 == 0 && k3 == 0) {
          coef[idx] = 0.0;
          continue;
        }
        double kv[3];
        for (int c = 0; c < 3; ++c)
          kv[c] = twoPi * (k1 * cell.rec[0][c] + k2 * cell.rec[1][c] + k3 * cell.rec[2][c]);
        double k2s = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
        if (k2s < kMinWavenumberSquared) {
          coef[idx] = 0.0;
          continue;
        }
        double mw = prefactor * std::exp(-k2s * inv4a2) / k2s;
        coef[idx] = mw * coef[idx];
      }
    }
  }
  std::vector<cplx> at(N);
  forward_nfft(N, t1.data(), t2.data(), t3.data(), M[0], M[1], M[2], m, coef.data(), at.data());
  for (int i = 0; i < N; ++i) pot[i] = at[i].real();
  if (!force) return;
  std::vector<cplx> deriv(nm);
  for (int c = 0; c < 3; ++c) {
    for (int a3 = 0; a3 < M[2]; ++a3) {
      int k3 = mode_of_bin(a3, M[2]);
      for (int a2 = 0; a2 < M[1]; ++a2) {
        int k2 = mode_of_bin(a2, M[1]);
        for (int a1 = 0; a1 < M[0]; ++a1) {
          int k1 = mode_of_bin(a1, M[0]);
          size_t idx = (static_cast<size_t>(a3) * M[1] + a2) * M[0] + a1;
          double kc = twoPi * (k1 * cell.rec[0][c] + k2 * cell.rec[1][c] + k3 * cell.rec[2][c]);
          deriv[idx] = cplx(0.0, kc) * coef[idx];
        }
      }
    }
    forward_nfft(N, t1.data(), t2.data(), t3.data(), M[0], M[1], M[2], m, deriv.data(), at.data());
    for (int i = 0; i < N; ++i) force[3 * i + c] = q[i] * at[i].real();
  }
}

// ----------------------------------------------------------------------------
// Direct engine splitting: common/ewald_alpha_search.f90:83-181 and
// direct/ewald_direct_3d.f90:319-347
// ----------------------------------------------------------------------------
double balanced_splitting(const Cell& cell, double tol) {
  const double minR = std::min(cell.latLen[0], std::min(cell.latLen[1], cell.latLen[2]));
  const double minG = 2.0 * kPi * std::min(cell.recLen[0], std::min(cell.recLen[1], cell.recLen[2]));
  const double V = cell.volume;
  auto cond = [&](double a) {
    double g4 = 4.0 * minG, g5 = 5.0 * minG;
    double f4 = (4.0 * kPi / V) * std::exp(-(g4 * g4) / (4.0 * (a * a))) / (g4 * g4);
    double f5 = (4.0 * kPi / V) * std::exp(-(g5 * g5) / (4.0 * (a * a))) / (g5 * g5);
    double r2 = 2.0 * minR, r3 = 3.0 * minR;
    return (f4 - f5) - (std::erfc(a * r2) / r2 - std::erfc(a * r3) / r3);
  };
  const double start = 1.0e-8;
  const double huge = std::numeric_limits<double>::max();
  int status = 0;
  double alpha = start;
  double imb = cond(alpha);
  while (imb < -tol && alpha <= huge) {
    alpha *= 2.0;
    imb = cond(alpha);
  }
  if (alpha > huge)
    status = 1;
  else if (alpha == start)
    status = 2;
  double left = 0.0, right = 0.0;
  if (status == 0) {
    left = 0.5 * alpha;
    while (imb < tol && alpha <= huge) {
      alpha *= 2.0;
      imb = cond(alpha);
    }
    if (alpha > huge) status = 3;
  }
  if (status == 0) {
    right = alpha;
    alpha = (left + right) / 2.0;
    int it = 0;
    imb = cond(alpha);
    while (std::fabs(imb) > tol && it <= 100) {
      if (imb < 0.0)
        left = alpha;
      else
        right = alpha;
      alpha = (left + right) / 2.0;
      imb = cond(alpha);
      ++it;
    }
    if (it > 100) status = 4;
  }
  if (status != 0) alpha = std::exp(-0.310104 * std::log(V) + 0.786382) / 2.0;
  return alpha;
}

// ----------------------------------------------------------------------------
// Stock DFTB+ Ewald stress: src/dftbp/dftb/coulomb.F90
// ----------------------------------------------------------------------------
double gTerm(double gg, double alpha, double vol) {  // :2713-2730
  return 4.0 * kPi * (std::exp(-0.25 * gg * gg / (alpha * alpha)) / (vol * gg * gg));
}
double rTerm(double rr, double alpha) { return std::erfc(alpha * rr) / rr; }  // :2734-2749

// getOptimalAlphaEwald, coulomb.F90:2097-2179
int optimal_alpha(double minG, double minR, double volume, double tol, double& alpha) {
  auto diff = [&](double a) {
    return (gTerm(4.0 * minG, a, volume) - gTerm(5.0 * minG, a, volume)) -
           (rTerm(2.0 * minR, a) - rTerm(3.0 * minR, a));
  };
  const double init = 1.0e-8, huge = std::numeric_limits<double>::max();
  int err = 0;
  alpha = init;
  double d = diff(alpha);
  while (d < -tol && alpha <= huge) {
    alpha *= 2.0;
    d = diff(alpha);
  }
  if (alpha > huge)
    err = 1;
  else if (alpha == init)
    err = 2;
  double left = 0.0, right = 0.0;
  if (err == 0) {
    left = 0.5 * alpha;
    while (d < tol && alpha <= huge) {
      alpha *= 2.0;
      d = diff(alpha);
    }
    if (alpha > huge) err = 3;
  }
  if (err == 0) {
    right = alpha;
    alpha = (left + right) / 2.0;
    int it = 0;
    d = diff(alpha);
    while (std::fabs(d) > tol && it <= kNSearchIter) {
      if (d < 0)
        left = alpha;
      else
        right = alpha;
      alpha = (left + right) / 2.0;
      d = diff(alpha);
      ++it;
    }
    if (it > kNSearchIter) err = 4;
  }
  return err == 0 ? EWO_OK : EWO_ERR_ALPHA_SEARCH;
}

// getMaxGEwald (:2183-2243) and getMaxREwald (:2249-2308): same bisection.
template <class F>
int max_extent(F term, double minValue, double& xx) {
  const double init = 1.0e-8, huge = std::numeric_limits<double>::max();
  int err = 0;
  xx = init;
  double yy = term(xx);
  while (yy > minValue && xx <= huge) {
    xx *= 2.0;
    yy = term(xx);
  }
  if (xx > huge)
    err = 1;
  else if (xx == init)
    err = 2;
  if (err == 0) {
    double xl = 0.5 * xx, yl = term(xl), xr = xx, yr = yy;
    int it = 1;
    while (yl - yr > minValue && it <= kNSearchIter) {
      xx = 0.5 * (xl + xr);
      yy = term(xx);
      if (yy >= minValue) {
        xl = xx;
        yl = yy;
      } else {
        xr = xx;
        yr = yy;
      }
      ++it;
    }
    if (it > kNSearchIter) err = 3;
  }
  return err == 0 ? EWO_OK : EWO_ERR_LATTICE_SEARCH;
}

// TLatPointIter with onlyInside, reduceByInversion, excludeOrigin
// (type/latpointiter.F90:62-273) as used by getLatticePoints
// (dftb/periodic.F90:272-336) in coulomb.F90:598-600.  basis[i][d] is basis
// vector i; invLen[i] = |inverse basis vector i|.
void lattice_points_half(const double basis[3][3], const double invLen[3], double dist,
                         std::vector<int>& pts) {
  int range[3];
  for (int i = 0; i < 3; ++i) range[i] = ffloor(dist * invLen[i]);
  const double cut2 = dist * dist;
  for (int c1 = 0; c1 <= range[0]; ++c1)
    for (int c2 = (c1 == 0 ? 0 : -range[1]); c2 <= range[1]; ++c2)
      for (int c3 = (c1 == 0 && c2 == 0 ? 0 : -range[2]); c3 <= range[2]; ++c3) {
        if (c1 == 0 && c2 == 0 && c3 == 0) continue;
        double rr[3];
        for (int d = 0; d < 3; ++d) rr[d] = c1 * basis[0][d] + c2 * basis[1][d] + c3 * basis[2][d];
        if (rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2] <= cut2) {
          pts.push_back(c1);
          pts.push_back(c2);
          pts.push_back(c3);
        }
      }
}

}  // namespace

// ============================================================================
// C entry points
// ============================================================================
extern "C" {

int ewo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

int ewo_next_fast_length(int n) { return next_fast_length(n); }
double ewo_lambert_w0(double x) { return lambert_w0(x); }

int ewo_fft3d(int n1, int n2, int n3, double* data, int isign) {
  fft3d(reinterpret_cast<cplx*>(data), n1, n2, n3, isign);
  return EWO_OK;
}

int ewo_adjoint_nfft(int n, const double* t1, const double* t2, const double* t3, const double* q,
                     int M1, int M2, int M3, int m, double* shat) {
  adjoint_nfft(n, t1, t2, t3, q, M1, M2, M3, m, reinterpret_cast<cplx*>(shat));
  return EWO_OK;
}

int ewo_forward_nfft(int n, const double* t1, const double* t2, const double* t3, int M1, int M2,
                     int M3, int m, const double* fhat, double* f) {
  forward_nfft(n, t1, t2, t3, M1, M2, M3, m, reinterpret_cast<const cplx*>(fhat),
               reinterpret_cast<cplx*>(f));
  return EWO_OK;
}

// ewald_parameters, fft/ewald_fft_3d.f90:142-191
int ewo_fft_parameters(int n, const double* charges, const double* lat, double tol,
                       const ewo_overrides* ov, ewo_params* out) {
  if (n <= 0) return EWO_ERR_NPARTICLE;
  Cell cell;
  int rc = cell_metrics(lat, cell);
  if (rc) return rc;
  double q2 = 0.0;
  for (int i = 0; i < n; ++i) q2 += charges[i] * charges[i];
  return choose_parameters(cell, q2, n, tol, ov, *out);
}

// ewald_grid_memory, fft/ewald_fft_3d.f90:197-244 with grid_memory_gigabytes,
// fft/ewald_fft_3d_parameters.f90:177-229
int ewo_fft_grid_memory(int n, const double* charges, const double* lat, double tol,
                        const ewo_overrides* ov, double* gigabytes) {
  ewo_params p;
  int rc = ewo_fft_parameters(n, charges, lat, tol, ov, &p);
  if (rc) return rc;
  double n1 = kOversampling * p.n_modes[0], n2 = kOversampling * p.n_modes[1],
         n3 = kOversampling * p.n_modes[2];
  double el = n1 * n2 * n3 + 2.0 * static_cast<double>(p.n_modes[0]) * p.n_modes[1] * p.n_modes[2];
  *gigabytes = el * 16.0 / (1024.0 * 1024.0 * 1024.0);
  return EWO_OK;
}

// ewald_potential_force, fft/ewald_fft_3d.f90:36-134
int ewo_fft_potential_force(int n, const double* positions, const double* charges, const double* lat,
                            double tol, double* pot, double* force, const ewo_overrides* ov) {
  int rc = check_configuration(n, positions, charges);
  if (rc) return rc;
  if (!pot || !lat) return EWO_ERR_ARG;
  Cell cell;
  rc = cell_metrics(lat, cell);
  if (rc) return rc;
  if (tol <= 0.0 || tol >= 1.0) return EWO_ERR_TOL;
  double q2 = 0.0;
  for (int i = 0; i < n; ++i) q2 += charges[i] * charges[i];
  ewo_params p;
  rc = choose_parameters(cell, q2, n, tol, ov, p);
  if (rc) return rc;
  std::vector<double> sp(n), lp(n), sf(3 * static_cast<size_t>(n)), lf(3 * static_cast<size_t>(n));
  for (double& t : g_stage_s) t = 0.0;
  {
    StageTimer t(ST_REAL);
    rc = short_range(n, positions, charges, cell, p.alpha, p.r_cut, sp.data(), sf.data(), nullptr);
  }
  if (rc) return rc;
  long_range(n, positions, charges, cell, p.alpha, p.n_modes, p.window_cutoff, lp.data(),
             force ? lf.data() : nullptr);
  for (int i = 0; i < n; ++i) pot[i] = sp[i] + lp[i] + (-2.0 * p.alpha / kSqrtPi * charges[i]);
  if (force)
    for (size_t k = 0; k < 3 * static_cast<size_t>(n); ++k) force[k] = sf[k] + lf[k];
  return EWO_OK;
}

int ewo_stage_seconds(double* out) {
  if (!out) return EWO_ERR_ARG;
  for (int i = 0; i < ST_N; ++i) out[i] = g_stage_s[i];
  return EWO_OK;
}

int ewo_real_space(int n, const double* positions, const double* charges, const double* lat,
                   double alpha, double r_cut, double* pot, double* force, int* used_cell_list) {
  Cell cell;
  int rc = cell_metrics(lat, cell);
  if (rc) return rc;
  return short_range(n, positions, charges, cell, alpha, r_cut, pot, force, used_cell_list);
}

// ewald_potential_force (direct), direct/ewald_direct_3d.f90:37-182
int ewo_direct_potential_force(int n, const double* positions, const double* charges,
                               const double* lat, double tol, double* pot, double* force,
                               const double* alpha_in, const double* r_cut_in,
                               const double* k_cut_in) {
  int rc = check_configuration(n, positions, charges);
  if (rc) return rc;
  Cell cell;
  rc = cell_metrics(lat, cell);
  if (rc) return rc;
  if (tol <= 0.0 || tol >= 1.0) return EWO_ERR_TOL;
  double alpha = alpha_in ? *alpha_in : balanced_splitting(cell, tol);
  if (alpha <= 0.0) return EWO_ERR_ALPHA;
  double r_cut = 0.0, k_cut = 0.0;
  if (!(r_cut_in && k_cut_in)) {
    r_cut = std::sqrt(-std::log(tol)) / alpha;  // direct_cutoffs, ewald_truncation.f90:36-45
    k_cut = 2.0 * alpha * std::sqrt(-std::log(tol));
  }
  if (r_cut_in) r_cut = *r_cut_in;
  if (k_cut_in) k_cut = *k_cut_in;
  if (r_cut <= 0.0 || k_cut <= 0.0) return EWO_ERR_CUTOFF;
  const double kc2 = k_cut * k_cut;
  rc = direct_real_space(n, positions, charges, cell, alpha, r_cut, pot, force);
  if (rc) return rc;
  int nM[3];
  for (int d = 0; d < 3; ++d) nM[d] = fceiling(k_cut * cell.latLen[d] / (2.0 * kPi)) + 1;
  std::vector<double> cs(n), sn(n);
  for (int mx = -nM[0]; mx <= nM[0]; ++mx)
    for (int my = -nM[1]; my <= nM[1]; ++my)
      for (int mz = -nM[2]; mz <= nM[2]; ++mz) {
        double kx = (mx * cell.rec[0][0] + my * cell.rec[1][0] + mz * cell.rec[2][0]) * 2.0 * kPi;
        double ky = (mx * cell.rec[0][1] + my * cell.rec[1][1] + mz * cell.rec[2][1]) * 2.0 * kPi;
        double kz = (mx * cell.rec[0][2] + my * cell.rec[1][2] + mz * cell.rec[2][2]) * 2.0 * kPi;
        double k2 = kx * kx + ky * ky + kz * kz;
        if (k2 < kMinWavenumberSquared) continue;
        if (k2 > kc2) continue;
        double mw = 4.0 * kPi / cell.volume * std::exp(-k2 / (4.0 * alpha * alpha)) / k2;
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < n; ++j) {
          double ph = kx * positions[j] + ky * positions[j + n] + kz * positions[j + 2 * n];
          cs[j] = std::cos(ph);
          sn[j] = std::sin(ph);
          sr += charges[j] * cs[j];
          si += charges[j] * sn[j];
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; ++i) {
          // S(k) exp(-i k.x_i)
          double lr = sr * cs[i] + si * sn[i];
          double li = si * cs[i] - sr * sn[i];
          pot[i] += mw * lr;
          if (force) {
            double ff = charges[i] * mw * li;
            force[3 * i] -= ff * kx;
            force[3 * i + 1] -= ff * ky;
            force[3 * i + 2] -= ff * kz;
          }
        }
      }
  for (int i = 0; i < n; ++i) pot[i] += -2.0 * alpha / kSqrtPi * charges[i];
  return EWO_OK;
}

// Stock stress: TCoulomb%updateLatVecs (coulomb.F90:575-620) then invRStress
// (coulomb.F90:2777-2863) with addNeighbourContribsStress (:2866-2905) over the
// dynamic neighbour list (type/dynneighlist.F90:178-298).
int ewo_stock_stress(int n, const double* coords, const double* dq, const double* lat_cols,
                     double tol_ewald, double alpha, double* stress_out, double* alpha_out,
                     double* max_r_out, double* max_g_out, int* n_g_out) {
  if (n <= 0) return EWO_ERR_NPARTICLE;
  // DFTB+ latVecs(:, i) = a_i; boundarycond.F90:433-438 for recVecs and volume.
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) a[i][d] = lat_cols[d + 3 * i];
  double c23[3], c31[3], c12[3];
  cross(a[1], a[2], c23);
  cross(a[2], a[0], c31);
  cross(a[0], a[1], c12);
  double det = a[0][0] * c23[0] + a[0][1] * c23[1] + a[0][2] * c23[2];
  double volume = std::fabs(det);
  if (volume <= kMinVolume) return EWO_ERR_VOLUME;
  double g[3][3];  // g[i] = 2 pi * inverse-transpose column i
  for (int d = 0; d < 3; ++d) {
    g[0][d] = 2.0 * kPi * c23[d] / det;
    g[1][d] = 2.0 * kPi * c31[d] / det;
    g[2][d] = 2.0 * kPi * c12[d] / det;
  }
  auto len = [](const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); };
  int rc;
  if (alpha <= 0.0) {
    double minG = std::min(len(g[0]), std::min(len(g[1]), len(g[2])));
    double minR = std::min(len(a[0]), std::min(len(a[1]), len(a[2])));
    rc = optimal_alpha(minG, minR, volume, tol_ewald, alpha);
    if (rc) return rc;
  }
  double maxR, maxG;
  rc = max_extent([&](double x) { return rTerm(x, alpha); }, tol_ewald, maxR);
  if (rc) return rc;
  rc = max_extent([&](double x) { return gTerm(x, alpha, volume); }, tol_ewald, maxG);
  if (rc) return rc;
  // Reciprocal half-space: basis = recVecs, inverse basis = latVecs/(2 pi).
  double invLenG[3] = {len(a[0]) / (2.0 * kPi), len(a[1]) / (2.0 * kPi), len(a[2]) / (2.0 * kPi)};
  std::vector<int> gp;
  lattice_points_half(g, invLenG, maxG, gp);
  const int nG = static_cast<int>(gp.size() / 3);
  double st[3][3] = {{0}};
  const double a2 = alpha * alpha;
  for (int ii = 0; ii < nG; ++ii) {
    double G[3];
    for (int d = 0; d < 3; ++d) G[d] = g[0][d] * gp[3 * ii] + g[1][d] * gp[3 * ii + 1] + g[2][d] * gp[3 * ii + 2];
    for (int inv = -1; inv <= 1; inv += 2) {
      double gv[3] = {inv * G[0], inv * G[1], inv * G[2]};
      double sc = 0.0, ss = 0.0;
#pragma omp parallel for reduction(+ : sc, ss) schedule(static)
      for (int i = 0; i < n; ++i) {
        double ph = gv[0] * coords[3 * i] + gv[1] * coords[3 * i + 1] + gv[2] * coords[3 * i + 2];
        sc += dq[i] * std::cos(ph);
        ss += dq[i] * std::sin(ph);
      }
      double im = sc * sc + ss * ss;
      double g2 = gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2];
      im = im * std::exp(-g2 / (4.0 * a2)) / g2;
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) {
          double t = (j == k ? 1.0 : 0.0) - 2.0 * (1.0 / (4.0 * a2) + 1.0 / g2) * gv[k] * gv[j];
          st[j][k] += t * im;
        }
    }
  }
  for (int j = 0; j < 3; ++j)
    for (int k = 0; k < 3; ++k) st[j][k] = -st[j][k] * 4.0 * kPi / volume;
  // Real space: half neighbour list at cutoff maxR.  Translations: all index
  // triples within floor(maxR |b_i|/(2 pi)) + 1, origin excluded.
  int rng[3];
  for (int i = 0; i < 3; ++i) rng[i] = ffloor(maxR * len(g[i]) / (2.0 * kPi)) + 1;
  std::vector<double> T;
  for (int c1 = -rng[0]; c1 <= rng[0]; ++c1)
    for (int c2 = -rng[1]; c2 <= rng[1]; ++c2)
      for (int c3 = -rng[2]; c3 <= rng[2]; ++c3) {
        if (c1 == 0 && c2 == 0 && c3 == 0) continue;
        for (int d = 0; d < 3; ++d) T.push_back(a[0][d] * c1 + a[1][d] * c2 + a[2][d] * c3);
      }
  const int nT = static_cast<int>(T.size() / 3);
  const double cut2 = maxR * maxR;
  double rs[9] = {0};
#pragma omp parallel
  {
    double loc[9] = {0};
#pragma omp for schedule(dynamic, 16)
    for (int i = 0; i < n; ++i) {
      const double* xi = coords + 3 * i;
      auto pair = [&](int j, const double* t, double scale) {
        double nc[3] = {coords[3 * j] + t[0], coords[3 * j + 1] + t[1], coords[3 * j + 2] + t[2]};
        double r[3] = {xi[0] - nc[0], xi[1] - nc[1], xi[2] - nc[2]};
        double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        if (d2 > cut2) return;
        double rr = std::sqrt(d2);
        double fac = alpha * rr;
        double dr = (-2.0 / std::sqrt(kPi) * std::exp(-fac * fac) * fac - std::erfc(fac)) / (rr * rr * rr);
        double f[3];
        for (int c = 0; c < 3; ++c) f[c] = r[c] * dr * dq[i] * dq[j];
        for (int ii = 0; ii < 3; ++ii)
          for (int jj = 0; jj < 3; ++jj) loc[jj + 3 * ii] += scale * (r[jj] * f[ii] + f[jj] * r[ii]);
      };
      const double zero[3] = {0.0, 0.0, 0.0};
      for (int j = i + 1; j < n; ++j) pair(j, zero, 1.0);
      for (int t = 0; t < nT; ++t)
        for (int j = i; j < n; ++j) pair(j, &T[3 * t], j == i ? 0.5 : 1.0);
    }
#pragma omp critical
    for (int k = 0; k < 9; ++k) rs[k] += loc[k];
  }
  for (int ii = 0; ii < 3; ++ii)
    for (int jj = 0; jj < 3; ++jj) stress_out[jj + 3 * ii] = (st[jj][ii] + rs[jj + 3 * ii]) / volume;
  if (alpha_out) *alpha_out = alpha;
  if (max_r_out) *max_r_out = maxR;
  if (max_g_out) *max_g_out = maxG;
  if (n_g_out) *n_g_out = nG;
  return EWO_OK;
}


}  // extern "C"

// ----------------------------------------------------------------------------
// Source -> target potentials and gradients with the stock Ewald sum:
// getPotential / getPotentialGradient / addExternalPotGrad (coulomb.F90:3122-3248)
// through sumInvRPeriodicAsymm (:1340-1418) and addInvRPrimePeriodicAsymm
// (:1934-2092), the pair function ewald (:2311-2343) with ewaldReciprocal
// (:2346-2386), ewaldReal (:2520-2575), derivEwaldReal (:2578-2625) and
// derivEwaldReciprocal (:2690-2711).  The lattice sums use updateLatVecs's
// setup (:575-620): the stock alpha, gLatPoints (half space, onlyInside) and the
// cell translations of getCellTranslations (dftb/periodic.F90:227-263).
// ----------------------------------------------------------------------------
namespace {

constexpr double kTolSameDist = 1.0e-5;  // common/accuracy.F90:69
constexpr double kTolSameDist2 = kTolSameDist * kTolSameDist;
constexpr double kErfArgLimit = 10.0;    // coulomb.F90:214

struct StockLattice {
  double alpha, volume;
  std::vector<double> R;  // Cartesian cell translations, origin first
  std::vector<double> G;  // Cartesian half-space reciprocal vectors
};

int stock_lattice(const double* lat_cols, double tol_ewald, double alpha, StockLattice& out) {
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) a[i][d] = lat_cols[d + 3 * i];
  double c23[3], c31[3], c12[3];
  cross(a[1], a[2], c23);
  cross(a[2], a[0], c31);
  cross(a[0], a[1], c12);
  const double det = a[0][0] * c23[0] + a[0][1] * c23[1] + a[0][2] * c23[2];
  const double volume = std::fabs(det);
  if (volume <= kMinVolume) return EWO_ERR_VOLUME;
  double g[3][3];
  for (int d = 0; d < 3; ++d) {
    g[0][d] = 2.0 * kPi * c23[d] / det;
    g[1][d] = 2.0 * kPi * c31[d] / det;
    g[2][d] = 2.0 * kPi * c12[d] / det;
  }
  auto len = [](const double* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); };
  int rc;
  if (alpha <= 0.0) {
    const double minG = std::min(len(g[0]), std::min(len(g[1]), len(g[2])));
    const double minR = std::min(len(a[0]), std::min(len(a[1]), len(a[2])));
    rc = optimal_alpha(minG, minR, volume, tol_ewald, alpha);
    if (rc) return rc;
  }
  double maxR, maxG;
  rc = max_extent([&](double x) { return rTerm(x, alpha); }, tol_ewald, maxR);
  if (rc) return rc;
  rc = max_extent([&](double x) { return gTerm(x, alpha, volume); }, tol_ewald, maxG);
  if (rc) return rc;
  const double invLenG[3] = {len(a[0]) / (2.0 * kPi), len(a[1]) / (2.0 * kPi),
                             len(a[2]) / (2.0 * kPi)};
  std::vector<int> gp;
  lattice_points_half(g, invLenG, maxG, gp);
  out.G.clear();
  for (size_t k = 0; k < gp.size(); k += 3)
    for (int d = 0; d < 3; ++d)
      out.G.push_back(g[0][d] * gp[k] + g[1][d] * gp[k + 1] + g[2][d] * gp[k + 2]);
  // getLatticePoints(latVecs, recVecs/(2 pi), maxR, posExtension=1, negExtension=1):
  // every index triple in [-(r_i + 1), r_i + 1], r_i = floor(maxR |b_i| / (2 pi)),
  // iterator order (last index fastest), with the origin moved to the front.
  int rng[3];
  for (int i = 0; i < 3; ++i) rng[i] = ffloor(maxR * len(g[i]) / (2.0 * kPi)) + 1;
  out.R.assign({0.0, 0.0, 0.0});
  for (int c1 = -rng[0]; c1 <= rng[0]; ++c1)
    for (int c2 = -rng[1]; c2 <= rng[1]; ++c2)
      for (int c3 = -rng[2]; c3 <= rng[2]; ++c3) {
        if (c1 == 0 && c2 == 0 && c3 == 0) continue;
        for (int d = 0; d < 3; ++d) out.R.push_back(a[0][d] * c1 + a[1][d] * c2 + a[2][d] * c3);
      }
  out.alpha = alpha;
  out.volume = volume;
  return EWO_OK;
}

// ewald(rr, rVec, gVec, alpha, vol, blurWidth, epsSoften), coulomb.F90:2311-2343
double ewald_pair(const double* rr, const StockLattice& L, double blur, double eps2) {
  const double alpha = L.alpha, vol = L.volume;
  // ewaldReciprocal: factor 2 for the half space
  double rec = 0.0;
  const double g2f = -1.0 / (4.0 * alpha * alpha);
  for (size_t k = 0; k < L.G.size(); k += 3) {
    const double* G = &L.G[k];
    const double g2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
    const double gr = G[0] * rr[0] + G[1] * rr[1] + G[2] * rr[2];
    rec += std::exp(g2f * g2) / g2 * std::cos(gr);
  }
  rec = 2.0 * rec * 4.0 * kPi / vol;
  // ewaldReal
  double real = 0.0;
  for (size_t k = 0; k < L.R.size(); k += 3) {
    const double x[3] = {rr[0] + L.R[k], rr[1] + L.R[k + 1], rr[2] + L.R[k + 2]};
    const double absRR = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    if (absRR < kTolSameDist * kTolSameDist) continue;
    const double r = std::sqrt(absRR), soft = std::sqrt(absRR + eps2);
    if (blur > 0.0) {
      real += (absRR < (kErfArgLimit * blur) * (kErfArgLimit * blur) ? std::erf(r / blur) : 1.0) /
              soft;
      real -= std::erf(alpha * r) / soft;
    } else {
      real += std::erfc(alpha * r) / soft;
    }
  }
  double e = rec + real - kPi / (vol * alpha * alpha);
  if (rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2] < kTolSameDist2) e -= 2.0 * alpha / std::sqrt(kPi);
  return e;
}

// derivEwaldReal + derivEwaldReciprocal, coulomb.F90:2578-2625, :2690-2711
void deriv_ewald_pair(const double* rr, const StockLattice& L, double blur, double* out) {
  const double alpha = L.alpha, vol = L.volume;
  double d[3] = {0.0, 0.0, 0.0};
  for (size_t k = 0; k < L.R.size(); k += 3) {
    const double x[3] = {rr[0] + L.R[k], rr[1] + L.R[k + 1], rr[2] + L.R[k + 2]};
    const double r = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    if (r < kTolSameDist2) continue;  // the reference compares r with tolSameDist**2 here
    double fac = alpha * r;
    double w = (-2.0 / std::sqrt(kPi) * std::exp(-fac * fac) * fac - std::erfc(fac)) / (r * r * r);
    if (blur > 0.0 && r < kErfArgLimit * blur) {
      fac = r / blur;
      w += (2.0 / std::sqrt(kPi) * std::exp(-fac * fac) * fac + std::erfc(fac)) / (r * r * r);
    }
    for (int c = 0; c < 3; ++c) d[c] += x[c] * w;
  }
  const double g2f = -1.0 / (4.0 * alpha * alpha);
  double g[3] = {0.0, 0.0, 0.0};
  for (size_t k = 0; k < L.G.size(); k += 3) {
    const double* G = &L.G[k];
    const double g2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
    const double gr = G[0] * rr[0] + G[1] * rr[1] + G[2] * rr[2];
    const double pf = -std::sin(gr) * std::exp(g2f * g2) / g2;
    for (int c = 0; c < 3; ++c) g[c] += pf * G[c];
  }
  for (int c = 0; c < 3; ++c) out[c] = d[c] + 2.0 * g[c] * 4.0 * kPi / vol;
}

}  // namespace

extern "C" {

int ewo_potential_at(int nt, const double* tcoords, int ns, const double* scoords,
                     const double* scharges, const double* blur, const double* eps_soften,
                     const double* lat_cols, double tol_ewald, double alpha, double* pot) {
  if (nt < 0 || ns < 0) return EWO_ERR_NPARTICLE;
  StockLattice L;
  const int rc = stock_lattice(lat_cols, tol_ewald, alpha, L);
  if (rc) return rc;
  const double eps2 = eps_soften ? (*eps_soften) * (*eps_soften) : 0.0;
#pragma omp parallel for schedule(dynamic, 4)
  for (int t = 0; t < nt; ++t) {
    double acc = 0.0;
    for (int s = 0; s < ns; ++s) {
      const double rr[3] = {tcoords[3 * t] - scoords[3 * s], tcoords[3 * t + 1] - scoords[3 * s + 1],
                            tcoords[3 * t + 2] - scoords[3 * s + 2]};
      acc += ewald_pair(rr, L, blur ? blur[s] : 0.0, eps2) * scharges[s];
    }
    pot[t] = acc;
  }
  return EWO_OK;
}

int ewo_potential_gradient_at(int nt, const double* tcoords, int ns, const double* scoords,
                              const double* scharges, const double* blur, const double* lat_cols,
                              double tol_ewald, double alpha, double* grad) {
  if (nt < 0 || ns < 0) return EWO_ERR_NPARTICLE;
  StockLattice L;
  const int rc = stock_lattice(lat_cols, tol_ewald, alpha, L);
  if (rc) return rc;
#pragma omp parallel for schedule(dynamic, 4)
  for (int t = 0; t < nt; ++t) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s < ns; ++s) {
      const double rr[3] = {tcoords[3 * t] - scoords[3 * s], tcoords[3 * t + 1] - scoords[3 * s + 1],
                            tcoords[3 * t + 2] - scoords[3 * s + 2]};
      double d[3];
      deriv_ewald_pair(rr, L, blur ? blur[s] : 0.0, d);
      for (int c = 0; c < 3; ++c) acc[c] += d[c] * scharges[s];
    }
    for (int c = 0; c < 3; ++c) grad[3 * t + c] = acc[c];
  }
  return EWO_OK;
}

int ewo_external_pot_grad(int na, const double* acoords, int ne, const double* ecoords,
                          const double* acharges, const double* echarges, int ham_deriv,
                          const double* eblur, const double* lat_cols, double tol_ewald,
                          double alpha, double* agrad, double* egrad) {
  if (na < 0 || ne < 0) return EWO_ERR_NPARTICLE;
  StockLattice L;
  const int rc = stock_lattice(lat_cols, tol_ewald, alpha, L);
  if (rc) return rc;
  std::vector<double> d0(3 * static_cast<size_t>(na), 0.0), d1(3 * static_cast<size_t>(ne), 0.0);
  for (int t = 0; t < na; ++t)
    for (int s = 0; s < ne; ++s) {
      const double rr[3] = {acoords[3 * t] - ecoords[3 * s], acoords[3 * t + 1] - ecoords[3 * s + 1],
                            acoords[3 * t + 2] - ecoords[3 * s + 2]};
      double d[3];
      deriv_ewald_pair(rr, L, eblur ? eblur[s] : 0.0, d);
      const double f = ham_deriv ? echarges[s] : acharges[t] * echarges[s];
      for (int c = 0; c < 3; ++c) {
        d0[3 * t + c] += d[c] * f;
        d1[3 * s + c] -= d[c] * f;
      }
    }
  for (size_t k = 0; k < d0.size(); ++k) agrad[k] += d0[k];
  if (!ham_deriv)
    for (size_t k = 0; k < d1.size(); ++k) egrad[k] += d1[k];
  return EWO_OK;
}


// XLBOMD gradient of the shadow energy with two charge sets,
// addInvRPrimeXlbomdPeriodic (coulomb.F90:1823-1894) with
// addNeighbourContribsXl (:1897-1930): over each atom pair and image within
// the stock cutoff maxR (the half neighbour list, self images skipped) and over
// all atom pairs in reciprocal space, prefac = qo_i qi_j + qi_i qo_j - qi_i qi_j
// times derivRTerm (:2752-2773) or derivEwaldReciprocal (:2690-2711).
int ewo_xlbomd_gradients(int n, const double* coords, const double* dq_in, const double* dq_out,
                         const double* lat_cols, double tol_ewald, double alpha, double* deriv) {
  if (n <= 0) return EWO_ERR_NPARTICLE;
  StockLattice L;
  int rc = stock_lattice(lat_cols, tol_ewald, alpha, L);
  if (rc) return rc;
  double maxR;
  rc = max_extent([&](double x) { return rTerm(x, L.alpha); }, tol_ewald, maxR);
  if (rc) return rc;
  const double cut2 = maxR * maxR;
  std::vector<double> loc(3 * static_cast<size_t>(n), 0.0);
  auto prefac = [&](int i, int j) {
    return dq_out[i] * dq_in[j] + dq_in[i] * dq_out[j] - dq_in[i] * dq_in[j];
  };
  // real space; L.R holds the origin first, then the other translations
  for (int i = 0; i < n; ++i)
    for (size_t t = 0; t < L.R.size(); t += 3)
      for (int j = i + 1; j < n; ++j) {
        const double rr[3] = {coords[3 * i] - coords[3 * j] - L.R[t],
                              coords[3 * i + 1] - coords[3 * j + 1] - L.R[t + 1],
                              coords[3 * i + 2] - coords[3 * j + 2] - L.R[t + 2]};
        const double d2 = rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2];
        if (d2 > cut2) continue;
        const double r = std::sqrt(d2), fac = L.alpha * r;
        const double w = prefac(i, j) *
                         (-2.0 * L.alpha / std::sqrt(kPi) * std::exp(-fac * fac) * r - std::erfc(fac)) /
                         (r * r * r);
        for (int c = 0; c < 3; ++c) {
          loc[3 * i + c] += w * rr[c];
          loc[3 * j + c] -= w * rr[c];
        }
      }
  // reciprocal space
  const double g2f = -1.0 / (4.0 * L.alpha * L.alpha);
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) {
      const double rr[3] = {coords[3 * i] - coords[3 * j], coords[3 * i + 1] - coords[3 * j + 1],
                            coords[3 * i + 2] - coords[3 * j + 2]};
      double g[3] = {0.0, 0.0, 0.0};
      for (size_t k = 0; k < L.G.size(); k += 3) {
        const double* G = &L.G[k];
        const double g2 = G[0] * G[0] + G[1] * G[1] + G[2] * G[2];
        const double pf = -std::sin(G[0] * rr[0] + G[1] * rr[1] + G[2] * rr[2]) *
                          std::exp(g2f * g2) / g2;
        for (int c = 0; c < 3; ++c) g[c] += pf * G[c];
      }
      const double p = prefac(i, j) * 2.0 * 4.0 * kPi / L.volume;
      for (int c = 0; c < 3; ++c) {
        loc[3 * i + c] += p * g[c];
        loc[3 * j + c] -= p * g[c];
      }
    }
  for (size_t k = 0; k < loc.size(); ++k) deriv[k] += loc[k];
  return EWO_OK;
}

}  // extern "C"
