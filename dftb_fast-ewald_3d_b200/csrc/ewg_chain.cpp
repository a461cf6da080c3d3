// ewg_chain.cpp -- host half of the Ewald operator: cell geometry, input
// validation, the reference's parameter chain and the stock DFTB+ setup of the
// stress.  All of it is O(1) or O(N) scalar work done once per call in FP64;
// the integer outputs (mode counts, window half-width, box counts) must match
// the reference exactly, so every expression keeps the reference's order of
// operations.  Paths are relative to the reference project.

#include <algorithm>
#include <cmath>
#include <limits>

#include "ewg_internal.h"

namespace ewg {
namespace {

constexpr double kMinVolume = 1.0e-18;            // common/ewald_geometry.f90:20
constexpr double kNeutralityTolerance = 1.0e-8;   // common/ewald_validation.f90:19
constexpr double kRealCutoffPrefactor = 3.0;      // fft/ewald_fft_3d_parameters.f90:16-18
constexpr double kRealBudgetFraction = 0.2;       // fft/ewald_fft_3d_parameters.f90:20-21
constexpr int kMinTransformLength = 4;            // nfft/fft_backend.f90:29
constexpr int kStockSearchIterations = 30;        // common/accuracy.F90:114 nSearchIter

double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

int finish_cell(Cell& cell) {
  double x23[3], x31[3], x12[3];
  cross3(cell.lat[1], cell.lat[2], x23);
  cross3(cell.lat[2], cell.lat[0], x31);
  cross3(cell.lat[0], cell.lat[1], x12);
  cell.volume = std::fabs(dot3(cell.lat[0], x23));
  if (!(cell.volume > kMinVolume)) return EWG_ERR_VOLUME;
  for (int d = 0; d < 3; ++d) {
    cell.rec[0][d] = x23[d] / cell.volume;
    cell.rec[1][d] = x31[d] / cell.volume;
    cell.rec[2][d] = x12[d] / cell.volume;
  }
  for (int i = 0; i < 3; ++i) {
    cell.latLen[i] = std::sqrt(dot3(cell.lat[i], cell.lat[i]));
    cell.recLen[i] = std::sqrt(dot3(cell.rec[i], cell.rec[i]));
  }
  return EWG_OK;
}

// lambert_w0 (common/ewald_lambert_w.f90:27-56): Halley iteration from log(1+x).
double lambert_w0(double x) {
  if (x <= 0.0) return 0.0;
  double w = std::log(1.0 + x);
  for (int it = 0; it < 60; ++it) {
    const double e = std::exp(w);
    const double f = w * e - x;
    const double w1 = w + 1.0;
    const double step = f / (e * w1 - 0.5 * (w + 2.0) * f / w1);
    w -= step;
    if (std::fabs(step) <= 1.0e-15 * (1.0 + std::fabs(w))) break;
  }
  return w;
}

int ceil_int(double x) { return static_cast<int>(std::ceil(x)); }
int floor_int(double x) { return static_cast<int>(std::floor(x)); }

}  // namespace

int cell_from_rows(const double* lat_rows, Cell& cell) {
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) cell.lat[i][d] = lat_rows[i + 3 * d];
  return finish_cell(cell);
}

int cell_from_cols(const double* lat_cols, Cell& cell) {
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) cell.lat[i][d] = lat_cols[d + 3 * i];
  return finish_cell(cell);
}

int check_sums(int n, double sum_q, double sum_abs_q) {
  if (n <= 0) return EWG_ERR_NPARTICLE;
  if (std::fabs(sum_q) > kNeutralityTolerance * sum_abs_q) return EWG_ERR_NOT_NEUTRAL;
  return EWG_OK;
}

int check_charges(int n, const double* q, double* q2sum, double* qsum) {
  if (n <= 0) return EWG_ERR_NPARTICLE;
  if (!q) return EWG_ERR_ARG;
  // One pass, three independent chains, each summed in index order.
  double s = 0.0, a = 0.0, s2 = 0.0;
  for (int i = 0; i < n; ++i) {
    const double v = q[i];
    s += v;
    a += std::fabs(v);
    s2 += v * v;
  }
  if (q2sum) *q2sum = s2;
  if (qsum) *qsum = s;
  return check_sums(n, s, a);
}

int next_fast_length(int n) {
  int len = n < 2 ? 2 : n;
  if (len & 1) ++len;
  for (;; len += 2) {
    int r = len;
    for (int p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) return len;
  }
}

double window_shape(int m) {
  const double s = static_cast<double>(kOversampling);
  return (2.0 * s / (2.0 * s - 1.0)) * (static_cast<double>(m) / kPi);
}

int box_count(double r_cut, double recLen) { return floor_int(1.0 / (r_cut * recLen)); }

int choose_parameters(const Cell& cell, double q2sum, int n, double tol, const ewg_overrides* ov,
                      ewg_params& p) {
  const ewg_overrides none{};
  const ewg_overrides& o = ov ? *ov : none;
  const double spacing = std::pow(cell.volume / static_cast<double>(n), 1.0 / 3.0);

  // 1. real-space cutoff (fft/ewald_fft_3d_parameters.f90:91-111)
  if (o.has_r_cut) {
    p.r_cut = o.r_cut;
  } else if (o.has_alpha) {
    p.r_cut = std::sqrt(-std::log(tol)) / o.alpha;
  } else {
    p.r_cut = kRealCutoffPrefactor * spacing;
    const double widest = std::max(std::max(cell.recLen[0], cell.recLen[1]), cell.recLen[2]);
    const double limit = 0.999 / (3.0 * widest);
    if (limit >= 1.5 * spacing) p.r_cut = std::min(p.r_cut, limit);
  }

  // 2. splitting parameter: splitting_from_real_budget (common/ewald_truncation.f90:53-78)
  if (o.has_alpha) {
    p.alpha = o.alpha;
  } else {
    const double budget = kRealBudgetFraction * tol;
    const double arg =
        (2.0 / budget) * q2sum * std::sqrt(p.r_cut / (static_cast<double>(n) * cell.volume));
    double w = arg > 0.0 ? lambert_w0(arg) : -std::log(budget);
    if (w <= 0.0) w = -std::log(budget);
    p.alpha = std::sqrt(w) / p.r_cut;
  }
  if (!(p.alpha > 0.0)) return EWG_ERR_ALPHA;

  // 3. Fourier cutoff: cutoff_from_fourier_budget (common/ewald_truncation.f90:84-104)
  {
    const double edge = std::pow(cell.volume, 1.0 / 3.0);
    const double arg = (4.0 / (3.0 * edge * edge)) *
                       std::pow(2.0 / (static_cast<double>(n) * p.alpha * kPi), 2.0 / 3.0) *
                       std::pow(2.0 * q2sum / tol, 4.0 / 3.0);
    double w = lambert_w0(arg);
    if (w <= 0.0) w = -std::log(tol);
    p.k_cut = std::sqrt(3.0) * p.alpha * std::sqrt(w);
  }
  if (o.has_k_cut) p.k_cut = o.k_cut;

  // 4. window half-width: window_cutoff_from_budget (nfft/nfft.f90:99-109)
  p.window_cutoff = std::max(2, ceil_int(std::log(4.0 / tol) / (2.0 * kPi / 3.0)));
  if (o.has_window_cutoff) p.window_cutoff = o.window_cutoff;

  // 5. modes per axis: modes_along_axis (fft/ewald_fft_3d_parameters.f90:152-168)
  for (int a = 0; a < 3; ++a) {
    const int highest = ceil_int(p.k_cut * cell.latLen[a] / (2.0 * kPi)) + 1;
    p.n_modes[a] = std::max(next_fast_length(2 * highest), kMinTransformLength);
  }
  if (o.has_n_modes)
    for (int a = 0; a < 3; ++a) p.n_modes[a] = o.n_modes;
  return EWG_OK;
}

double grid_memory_gigabytes(const ewg_params& p) {
  const double n1 = kOversampling * p.n_modes[0], n2 = kOversampling * p.n_modes[1],
               n3 = kOversampling * p.n_modes[2];
  const double modes = static_cast<double>(p.n_modes[0]) * p.n_modes[1] * p.n_modes[2];
  return (n1 * n2 * n3 + 2.0 * modes) * 16.0 / (1024.0 * 1024.0 * 1024.0);
}

double balanced_splitting(const Cell& cell, double tol) {
  // balanced_alpha (common/ewald_alpha_search.f90:83-181) on the shortest
  // lattice and reciprocal vectors; volume fit when no bracket exists.
  const double minR = std::min(std::min(cell.latLen[0], cell.latLen[1]), cell.latLen[2]);
  const double minG =
      2.0 * kPi * std::min(std::min(cell.recLen[0], cell.recLen[1]), cell.recLen[2]);
  const double V = cell.volume;
  auto imbalance = [&](double a) {
    const double g4 = 4.0 * minG, g5 = 5.0 * minG;
    const double f4 = (4.0 * kPi / V) * std::exp(-(g4 * g4) / (4.0 * (a * a))) / (g4 * g4);
    const double f5 = (4.0 * kPi / V) * std::exp(-(g5 * g5) / (4.0 * (a * a))) / (g5 * g5);
    const double r2 = 2.0 * minR, r3 = 3.0 * minR;
    return (f4 - f5) - (std::erfc(a * r2) / r2 - std::erfc(a * r3) / r3);
  };
  const double start = 1.0e-8, big = std::numeric_limits<double>::max();
  bool ok = true;
  double a = start, f = imbalance(a);
  while (f < -tol && a <= big) f = imbalance(a *= 2.0);
  if (a > big || a == start) ok = false;
  double lo = 0.0, hi = 0.0;
  if (ok) {
    lo = 0.5 * a;
    while (f < tol && a <= big) f = imbalance(a *= 2.0);
    if (a > big) ok = false;
  }
  if (ok) {
    hi = a;
    a = (lo + hi) / 2.0;
    f = imbalance(a);
    int it = 0;
    while (std::fabs(f) > tol && it <= 100) {
      (f < 0.0 ? lo : hi) = a;
      a = (lo + hi) / 2.0;
      f = imbalance(a);
      ++it;
    }
    if (it > 100) ok = false;
  }
  if (!ok) a = std::exp(-0.310104 * std::log(V) + 0.786382) / 2.0;
  return a;
}

namespace {
// gTerm / rTerm (coulomb.F90:2713-2749)
double g_term(double g, double alpha, double V) {
  return 4.0 * kPi * (std::exp(-0.25 * g * g / (alpha * alpha)) / (V * g * g));
}
double r_term(double r, double alpha) { return std::erfc(alpha * r) / r; }

// Bisection shared by getMaxGEwald (coulomb.F90:2183-2243) and getMaxREwald
// (:2249-2308): double until the term drops below minValue, then halve the
// bracket at most nSearchIter times.
template <class Term>
int largest_significant(Term term, double minValue, double& x) {
  const double start = 1.0e-8, big = std::numeric_limits<double>::max();
  x = start;
  double y = term(x);
  while (y > minValue && x <= big) y = term(x *= 2.0);
  if (x > big || x == start) return EWG_ERR_LATTICE_SEARCH;
  double xl = 0.5 * x, yl = term(xl), xr = x, yr = y;
  int it = 1;
  while (yl - yr > minValue && it <= kStockSearchIterations) {
    x = 0.5 * (xl + xr);
    y = term(x);
    if (y >= minValue) {
      xl = x;
      yl = y;
    } else {
      xr = x;
      yr = y;
    }
    ++it;
  }
  return it > kStockSearchIterations ? EWG_ERR_LATTICE_SEARCH : EWG_OK;
}
}  // namespace

int stock_setup(const Cell& cell, double tol, double alpha_in, StockSetup& out) {
  // Reciprocal vectors with the factor 2 pi, as DFTB+ stores them
  // (dftb/boundarycond.F90:433-438).
  double G[3][3];
  for (int i = 0; i < 3; ++i)
    for (int d = 0; d < 3; ++d) G[i][d] = 2.0 * kPi * cell.rec[i][d];
  double alpha = alpha_in;
  if (!(alpha > 0.0)) {
    // getOptimalAlphaEwald (coulomb.F90:2097-2179)
    const double minG = 2.0 * kPi * std::min(std::min(cell.recLen[0], cell.recLen[1]), cell.recLen[2]);
    const double minR = std::min(std::min(cell.latLen[0], cell.latLen[1]), cell.latLen[2]);
    const double V = cell.volume;
    auto diff = [&](double a) {
      return (g_term(4.0 * minG, a, V) - g_term(5.0 * minG, a, V)) -
             (r_term(2.0 * minR, a) - r_term(3.0 * minR, a));
    };
    const double start = 1.0e-8, big = std::numeric_limits<double>::max();
    alpha = start;
    double d = diff(alpha);
    while (d < -tol && alpha <= big) d = diff(alpha *= 2.0);
    if (alpha > big || alpha == start) return EWG_ERR_ALPHA_SEARCH;
    double lo = 0.5 * alpha;
    while (d < tol && alpha <= big) d = diff(alpha *= 2.0);
    if (alpha > big) return EWG_ERR_ALPHA_SEARCH;
    double hi = alpha;
    alpha = (lo + hi) / 2.0;
    d = diff(alpha);
    int it = 0;
    while (std::fabs(d) > tol && it <= kStockSearchIterations) {
      (d < 0 ? lo : hi) = alpha;
      alpha = (lo + hi) / 2.0;
      d = diff(alpha);
      ++it;
    }
    if (it > kStockSearchIterations) return EWG_ERR_ALPHA_SEARCH;
  }
  out.alpha = alpha;
  int rc = largest_significant([&](double r) { return r_term(r, alpha); }, tol, out.max_r);
  if (rc) return rc;
  rc = largest_significant([&](double g) { return g_term(g, alpha, cell.volume); }, tol, out.max_g);
  if (rc) return rc;
  // getLatticePoints(recVecs, latVecs/(2 pi), maxG, onlyInside, reduceByInversion,
  // withoutOrigin) (dftb/periodic.F90:272-336, type/latpointiter.F90:62-273):
  // half space (c1 > 0, or c1 = 0 and c2 > 0, or c1 = c2 = 0 and c3 > 0) inside maxG.
  int range[3];
  for (int i = 0; i < 3; ++i) range[i] = floor_int(out.max_g * (cell.latLen[i] / (2.0 * kPi)));
  const double cut2 = out.max_g * out.max_g;
  out.g.clear();
  for (int c1 = 0; c1 <= range[0]; ++c1)
    for (int c2 = (c1 == 0 ? 0 : -range[1]); c2 <= range[1]; ++c2)
      for (int c3 = (c1 == 0 && c2 == 0 ? 0 : -range[2]); c3 <= range[2]; ++c3) {
        if (c1 == 0 && c2 == 0 && c3 == 0) continue;
        double v[3];
        for (int d = 0; d < 3; ++d) v[d] = c1 * G[0][d] + c2 * G[1][d] + c3 * G[2][d];
        if (dot3(v, v) <= cut2) out.g.insert(out.g.end(), v, v + 3);
      }
  return EWG_OK;
}

}  // namespace ewg
