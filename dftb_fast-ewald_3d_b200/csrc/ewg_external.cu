// ewg_external.cu -- potentials and gradients at arbitrary points from a set of
// point charges, with the stock Ewald sum of DFTB+'s TCoulomb:
// getPotential / getPotentialGradient / addExternalPotGrad
// (dftb/coulomb.F90:3122-3248) through sumInvRPeriodicAsymm (:1340-1418) and
// addInvRPrimePeriodicAsymm (:1934-2092).
//
// Per (target, source) pair the reference evaluates the pair function ewald
// (:2311-2343): the real-space sum over the cell translations (ewaldReal
// :2520-2575, with the Gaussian blur of the source and the softening), the
// reciprocal sum over the half-space G vectors (ewaldReciprocal :2346-2386), the
// constant -pi/(V alpha^2) and, for coincident points, -2 alpha/sqrt(pi).
//
// On the GPU one warp takes one target (or one source for the source-side
// gradient) and its lanes stride over the other group.  The reciprocal sum is
// regrouped through the other group's structure factors,
//   sum_s q_s cos(G.(r_t - r_s)) = cos(G.r_t) C(G) + sin(G.r_t) S(G),
// C = sum_s q_s cos(G.r_s), S = sum_s q_s sin(G.r_s), an exact identity that
// turns O(N_t N_s N_G) work into O((N_t + N_s) N_G).  Sums run in a fixed order
// (lane-strided, then a fixed shuffle tree): results are reproducible.

#include <cuda_runtime.h>

#include "ewg_kernels.h"

namespace ewg {

namespace {

constexpr double kTolSameDist = 1.0e-5;  // common/accuracy.F90:69
constexpr double kErfArgLimit = 10.0;    // coulomb.F90:214
constexpr double kSqrtPiExt = 1.77245385090551602730;

__device__ __forceinline__ double warp_sum_ext(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// ewaldReal (coulomb.F90:2520-2575); blur <= 0 means no blur.
__device__ __forceinline__ double real_pot(const double* rr, const ExtLattice& L, double blur,
                                           double eps2) {
  double sum = 0.0;
  for (int k = 0; k < L.nR; ++k) {
    const double x0 = rr[0] + L.R[3 * k], x1 = rr[1] + L.R[3 * k + 1], x2 = rr[2] + L.R[3 * k + 2];
    const double absRR = x0 * x0 + x1 * x1 + x2 * x2;
    if (absRR < kTolSameDist * kTolSameDist) continue;
    const double r = sqrt(absRR), soft = sqrt(absRR + eps2);
    if (blur > 0.0) {
      const double lim = kErfArgLimit * blur;
      sum += (absRR < lim * lim ? erf(r / blur) : 1.0) / soft;
      sum -= erf(L.alpha * r) / soft;
    } else {
      sum += erfc(L.alpha * r) / soft;
    }
  }
  return sum;
}

// derivEwaldReal (coulomb.F90:2578-2625).  The reference skips terms with
// r < tolSameDist**2 here (a distance compared with a squared tolerance).
__device__ __forceinline__ void real_deriv(const double* rr, const ExtLattice& L, double blur,
                                           double* out) {
  double d0 = 0.0, d1 = 0.0, d2 = 0.0;
  for (int k = 0; k < L.nR; ++k) {
    const double x0 = rr[0] + L.R[3 * k], x1 = rr[1] + L.R[3 * k + 1], x2 = rr[2] + L.R[3 * k + 2];
    const double r = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
    if (r < kTolSameDist * kTolSameDist) continue;
    double fac = L.alpha * r;
    const double r3 = r * r * r;
    double w = (-2.0 / kSqrtPiExt * exp(-fac * fac) * fac - erfc(fac)) / r3;
    if (blur > 0.0 && r < kErfArgLimit * blur) {
      fac = r / blur;
      w += (2.0 / kSqrtPiExt * exp(-fac * fac) * fac + erfc(fac)) / r3;
    }
    d0 += x0 * w;
    d1 += x1 * w;
    d2 += x2 * w;
  }
  out[0] = d0;
  out[1] = d1;
  out[2] = d2;
}

// Potential at each target (sumInvRPeriodicAsymm).  L.sf holds the sources'
// structure factors.  const_term = -pi/(V alpha^2) * sum_s q_s.
__global__ void __launch_bounds__(256) k_ext_potential(int nt, const double* __restrict__ tc,
                                                       int ns, const double* __restrict__ sc,
                                                       const double* __restrict__ sq,
                                                       const double* __restrict__ blur,
                                                       double eps2, ExtLattice L,
                                                       double const_term,
                                                       double* __restrict__ pot) {
  const int t = static_cast<int>((static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= nt) return;
  const double rt[3] = {tc[3 * t], tc[3 * t + 1], tc[3 * t + 2]};
  const double self = 2.0 * L.alpha / kSqrtPiExt;
  double acc = 0.0;
  for (int s = lane; s < ns; s += 32) {
    const double rr[3] = {rt[0] - sc[3 * s], rt[1] - sc[3 * s + 1], rt[2] - sc[3 * s + 2]};
    double v = real_pot(rr, L, blur ? blur[s] : 0.0, eps2);
    if (rr[0] * rr[0] + rr[1] * rr[1] + rr[2] * rr[2] < kTolSameDist * kTolSameDist) v -= self;
    acc += v * sq[s];
  }
  const double rec = 2.0 * 4.0 * 3.14159265358979323846 / L.volume;
  const double g2f = -1.0 / (4.0 * L.alpha * L.alpha);
  for (int g = lane; g < L.nG; g += 32) {
    const double G0 = L.G[3 * g], G1 = L.G[3 * g + 1], G2 = L.G[3 * g + 2];
    const double g2 = G0 * G0 + G1 * G1 + G2 * G2;
    double sn, cs;
    sincos(G0 * rt[0] + G1 * rt[1] + G2 * rt[2], &sn, &cs);
    acc += rec * exp(g2f * g2) / g2 * (cs * L.sf[2 * g] + sn * L.sf[2 * g + 1]);
  }
  acc = warp_sum_ext(acc);
  if (lane == 0) pot[t] = acc + const_term;
}

// Gradient at each target (addInvRPrimePeriodicAsymm, group 0), optionally
// scaled per target (scale = q_t for the force form) and added to `grad`.
__global__ void __launch_bounds__(256) k_ext_gradient(int nt, const double* __restrict__ tc,
                                                      int ns, const double* __restrict__ sc,
                                                      const double* __restrict__ sq,
                                                      const double* __restrict__ blur,
                                                      ExtLattice L,
                                                      const double* __restrict__ scale,
                                                      double* __restrict__ grad) {
  const int t = static_cast<int>((static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= nt) return;
  const double rt[3] = {tc[3 * t], tc[3 * t + 1], tc[3 * t + 2]};
  double acc[3] = {0.0, 0.0, 0.0};
  for (int s = lane; s < ns; s += 32) {
    const double rr[3] = {rt[0] - sc[3 * s], rt[1] - sc[3 * s + 1], rt[2] - sc[3 * s + 2]};
    double d[3];
    real_deriv(rr, L, blur ? blur[s] : 0.0, d);
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] += d[c] * sq[s];
  }
  // sum_s q_s (-sin(G.(r_t - r_s))) = -(sin(G.r_t) C - cos(G.r_t) S)
  const double rec = 2.0 * 4.0 * 3.14159265358979323846 / L.volume;
  const double g2f = -1.0 / (4.0 * L.alpha * L.alpha);
  for (int g = lane; g < L.nG; g += 32) {
    const double G0 = L.G[3 * g], G1 = L.G[3 * g + 1], G2 = L.G[3 * g + 2];
    const double g2 = G0 * G0 + G1 * G1 + G2 * G2;
    double sn, cs;
    sincos(G0 * rt[0] + G1 * rt[1] + G2 * rt[2], &sn, &cs);
    const double pf = -rec * exp(g2f * g2) / g2 * (sn * L.sf[2 * g] - cs * L.sf[2 * g + 1]);
    acc[0] += pf * G0;
    acc[1] += pf * G1;
    acc[2] += pf * G2;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) acc[c] = warp_sum_ext(acc[c]);
  if (lane == 0) {
    const double f = scale ? scale[t] : 1.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) grad[3 * t + c] += f * acc[c];
  }
}

// Source-side gradient of the force form (addInvRPrimePeriodicAsymm, group 1):
// grad_s -= q_s sum_t q_t d(r_t - r_s), one warp per source; L.sf holds the
// targets' structure factors.
__global__ void __launch_bounds__(256) k_ext_source_gradient(int nt, const double* __restrict__ tc,
                                                             const double* __restrict__ tq, int ns,
                                                             const double* __restrict__ sc,
                                                             const double* __restrict__ sq,
                                                             const double* __restrict__ blur,
                                                             ExtLattice L,
                                                             double* __restrict__ grad) {
  const int s = static_cast<int>((static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (s >= ns) return;
  const double rs[3] = {sc[3 * s], sc[3 * s + 1], sc[3 * s + 2]};
  const double bs = blur ? blur[s] : 0.0;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int t = lane; t < nt; t += 32) {
    const double rr[3] = {tc[3 * t] - rs[0], tc[3 * t + 1] - rs[1], tc[3 * t + 2] - rs[2]};
    double d[3];
    real_deriv(rr, L, bs, d);
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] += d[c] * tq[t];
  }
  // sum_t q_t (-sin(G.(r_t - r_s))) = -(S_t cos(G.r_s) - C_t sin(G.r_s))
  const double rec = 2.0 * 4.0 * 3.14159265358979323846 / L.volume;
  const double g2f = -1.0 / (4.0 * L.alpha * L.alpha);
  for (int g = lane; g < L.nG; g += 32) {
    const double G0 = L.G[3 * g], G1 = L.G[3 * g + 1], G2 = L.G[3 * g + 2];
    const double g2 = G0 * G0 + G1 * G1 + G2 * G2;
    double sn, cs;
    sincos(G0 * rs[0] + G1 * rs[1] + G2 * rs[2], &sn, &cs);
    const double pf = -rec * exp(g2f * g2) / g2 * (L.sf[2 * g + 1] * cs - L.sf[2 * g] * sn);
    acc[0] += pf * G0;
    acc[1] += pf * G1;
    acc[2] += pf * G2;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) acc[c] = warp_sum_ext(acc[c]);
  if (lane == 0) {
#pragma unroll
    for (int c = 0; c < 3; ++c) grad[3 * s + c] -= sq[s] * acc[c];
  }
}

inline int warp_blocks(long n) { return static_cast<int>((32 * n + 255) / 256); }

}  // namespace

void launch_ext_potential(int nt, const double* tc, int ns, const double* sc, const double* sq,
                          const double* blur, double eps2, const ExtLattice& L, double const_term,
                          double* pot, cudaStream_t st) {
  if (nt == 0) return;
  k_ext_potential<<<warp_blocks(nt), 256, 0, st>>>(nt, tc, ns, sc, sq, blur, eps2, L, const_term,
                                                   pot);
  ++g_launches;
}

void launch_ext_gradient(int nt, const double* tc, int ns, const double* sc, const double* sq,
                         const double* blur, const ExtLattice& L, const double* scale,
                         double* grad, cudaStream_t st) {
  if (nt == 0) return;
  k_ext_gradient<<<warp_blocks(nt), 256, 0, st>>>(nt, tc, ns, sc, sq, blur, L, scale, grad);
  ++g_launches;
}

void launch_ext_source_gradient(int nt, const double* tc, const double* tq, int ns,
                                const double* sc, const double* sq, const double* blur,
                                const ExtLattice& L, double* grad, cudaStream_t st) {
  if (ns == 0) return;
  k_ext_source_gradient<<<warp_blocks(ns), 256, 0, st>>>(nt, tc, tq, ns, sc, sq, blur, L, grad);
  ++g_launches;
}

}  // namespace ewg
