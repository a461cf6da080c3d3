// ewg_points.cu -- the real-space half of the mesh-based potentials and
// gradients at arbitrary points (targets) from a set of point charges
// (sources): TCoulomb getPotential / getPotentialGradient / addExternalPotGrad
// (dftb/coulomb.F90:3122-3248) at a cost linear in the number of points.
//
// The stock routines evaluate the pair function ewald (:2311-2343) for every
// (target, source) pair with DFTB+'s own splitting, whose real-space part
// reaches hundreds of Bohr in large cells.  The pair function is a periodic
// Ewald sum, independent of the splitting alpha: for a source of Gaussian
// width w (blur) it is
//   sum_R [erf(r/w) - erf(alpha r)] / r  +  (4 pi / V) sum_G e^{-G^2/4alpha^2}/G^2 cos(G.r)
//   - pi / (V alpha^2)   [- 2 alpha / sqrt(pi) for coincident points]
// (erf(r/w) -> 1 without blur).  The mesh form takes alpha from the fast
// path's parameter chain: the Fourier sum runs through the NFFT (spread the
// sources, influence weights, gather at the targets), and the real-space sum
// below runs over a cell list of the sources, keeping the pairs within the
// chain's cutoff (widened to cover the widest blur).  The terms follow the
// reference's ewaldReal (:2520-2575) and derivEwaldReal (:2578-2625) one to
// one, including which coincident images they skip.
//
// One warp per target; its lanes take the neighbour boxes of the target's box
// (periodic images included, so cells narrower than the cutoff work too) and
// walk the sources of each box.  Lane sums then a fixed shuffle tree: results
// are reproducible.

#include <cuda_runtime.h>

#include "ewg_kernels.h"

namespace ewg {

namespace {

constexpr double kTolSameDistP = 1.0e-5;  // common/accuracy.F90:69
constexpr double kErfArgLimitP = 10.0;    // coulomb.F90:214
constexpr double kSqrtPiP = 1.77245385090551602730;

__device__ __forceinline__ double warp_sum_pts(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

__device__ __forceinline__ int floor_div(int a, int b) {
  const int q = a / b;
  return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}

__global__ void __launch_bounds__(256) k_points_real(
    int nt, const double* __restrict__ tc, const double* __restrict__ tblur, int ns,
    const double4* __restrict__ s4s, const int* __restrict__ sperm,
    const double* __restrict__ sc, const double* __restrict__ sblur,
    const int* __restrict__ box_start, PointsReal g, double* __restrict__ pot,
    double* __restrict__ grad) {
  const int t = static_cast<int>((static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= nt) return;  // whole warps leave together
  const double x[3] = {tc[3 * t], tc[3 * t + 1], tc[3 * t + 2]};
  double st[3];
  int bt[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double u = g.rec[d][0] * x[0] + g.rec[d][1] * x[1] + g.rec[d][2] * x[2];
    st[d] = u - floor(u);
    bt[d] = min(static_cast<int>(st[d] * g.nb[d]), g.nb[d] - 1);
  }
  const double wt = tblur ? tblur[t] : 0.0;
  const int sx = 2 * g.R[0] + 1, sy = 2 * g.R[1] + 1;
  const int nbox = sx * sy * (2 * g.R[2] + 1);
  const double self = 2.0 * g.alpha / kSqrtPiP;
  double p = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
  for (int b = lane; b < nbox; b += 32) {
    const int o[3] = {b % sx - g.R[0], (b / sx) % sy - g.R[1], b / (sx * sy) - g.R[2]};
    int box[3];
    double shift[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int raw = bt[d] + o[d];
      const int wrap = floor_div(raw, g.nb[d]);
      box[d] = raw - wrap * g.nb[d];
      shift[d] = static_cast<double>(wrap);
    }
    const int key = (box[2] * g.nb[1] + box[1]) * g.nb[0] + box[0];
    const int k1 = box_start[key + 1];
    for (int k = box_start[key]; k < k1; ++k) {
      const double4 s = s4s[k];
      const double f[3] = {st[0] - (s.x + shift[0]), st[1] - (s.y + shift[1]),
                           st[2] - (s.z + shift[2])};
      double r[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) r[c] = f[0] * g.lat[0][c] + f[1] * g.lat[1][c] + f[2] * g.lat[2][c];
      const double rr2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      if (rr2 > g.r_cut2) continue;
      const int i = sperm[k];
      const double w = sblur ? sblur[i] : wt;
      const double qs = s.w;
      const double rr = sqrt(rr2);
      if (g.want_pot) {
        if (rr2 < kTolSameDistP * kTolSameDistP) {
          // ewaldReal skips the coincident image; ewald subtracts the self
          // term when the two points themselves (not an image) coincide.
          const double d0 = x[0] - sc[3 * i], d1 = x[1] - sc[3 * i + 1], d2 = x[2] - sc[3 * i + 2];
          if (d0 * d0 + d1 * d1 + d2 * d2 < kTolSameDistP * kTolSameDistP) p -= self * qs;
        } else if (w > 0.0) {
          const double lim = kErfArgLimitP * w;
          p += qs * (((rr2 < lim * lim) ? erf(rr / w) : 1.0) / rr - erf(g.alpha * rr) / rr);
        } else {
          p += qs * erfc(g.alpha * rr) / rr;
        }
      }
      // derivEwaldReal skips r < tolSameDist**2 (a distance against a squared
      // tolerance, as the reference writes it).
      if (g.want_grad && rr >= kTolSameDistP * kTolSameDistP) {
        double fac = g.alpha * rr;
        const double r3 = rr * rr2;
        double dw = (-2.0 / kSqrtPiP * exp(-fac * fac) * fac - erfc(fac)) / r3;
        if (w > 0.0 && rr < kErfArgLimitP * w) {
          fac = rr / w;
          dw += (2.0 / kSqrtPiP * exp(-fac * fac) * fac + erfc(fac)) / r3;
        }
        dw *= qs;
        g0 += r[0] * dw;
        g1 += r[1] * dw;
        g2 += r[2] * dw;
      }
    }
  }
  if (g.want_pot) {
    p = warp_sum_pts(p);
    if (lane == 0) pot[t] = p;
  }
  if (g.want_grad) {
    g0 = warp_sum_pts(g0);
    g1 = warp_sum_pts(g1);
    g2 = warp_sum_pts(g2);
    if (lane == 0) {
      grad[3 * t] = g0;
      grad[3 * t + 1] = g1;
      grad[3 * t + 2] = g2;
    }
  }
}

__global__ void k_fill(double* __restrict__ x, int n, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = v;
}

__global__ void k_add_scaled3(int n, const double* __restrict__ scale,
                              const double* __restrict__ src, double* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * n) return;
  dst[i] += (scale ? scale[i / 3] : 1.0) * src[i];
}

}  // namespace

void launch_points_real(int nt, const double* tc, const double* tblur, int ns, const double4* s4s,
                        const int* sperm, const double* sc, const double* sblur,
                        const int* box_start, const PointsReal& g, double* pot, double* grad,
                        cudaStream_t st) {
  if (nt == 0) return;
  const long threads = 32L * nt;
  k_points_real<<<static_cast<unsigned>((threads + 255) / 256), 256, 0, st>>>(
      nt, tc, tblur, ns, s4s, sperm, sc, sblur, box_start, g, pot, grad);
  ++g_launches;
}

void launch_fill(double* x, int n, double v, cudaStream_t st) {
  if (n == 0) return;
  k_fill<<<(n + 255) / 256, 256, 0, st>>>(x, n, v);
  ++g_launches;
}

void launch_add_scaled3(int n, const double* scale, const double* src, double* dst,
                        cudaStream_t st) {
  if (n == 0) return;
  k_add_scaled3<<<(3 * n + 255) / 256, 256, 0, st>>>(n, scale, src, dst);
  ++g_launches;
}

}  // namespace ewg
